"""Builds libterawarp_b200.so (sm_100a) in-tree with nvcc.

The library is a plain C ABI (include/terawarp_b200.h); it is compiled
directly with nvcc, not as a torch extension, so its signatures carry no
torch types.  Output: terawarp_b200/libterawarp_b200.so, and the command-line front end
terawarp_b200/terawarp (cli/tw_main.cpp) linked against it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "libterawarp_b200.so"
CLI_SRC = PKG / "cli" / "tw_main.cpp"
CLI = PKG / "terawarp"
BUILD = PKG / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = Path(cuda) / "bin" / "nvcc"
    return str(p) if p.exists() else (shutil.which("nvcc") or "nvcc")


def _host_cxx() -> str:
    # the environment's CC/CXX may point at a compiler without OpenMP/libstdc++ extras
    return shutil.which("g++") or "g++"


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    cmd = [_nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", _host_cxx(),
           "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build_cli() -> Path:
    """The terawarp executable: tw_main.cpp against the library (rpath = its own directory)."""
    cmd = [_host_cxx(), "-O2", "-std=c++17", "-I", str(ROOT / "include"), str(CLI_SRC), "-L", str(PKG),
           "-lterawarp_b200", "-Wl,-rpath,$ORIGIN", "-o", str(CLI) + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building the terawarp command failed:\n{r.stdout}\n{r.stderr}")
    os.replace(str(CLI) + ".tmp", CLI)
    return CLI


def build(force: bool = False, verbose: bool = False) -> Path:
    srcs = sources()
    headers = list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    newest = max(p.stat().st_mtime for p in srcs + headers + [Path(__file__)])
    if OUT.exists() and not force and OUT.stat().st_mtime >= newest:
        if not CLI.exists() or CLI.stat().st_mtime < max(OUT.stat().st_mtime, CLI_SRC.stat().st_mtime):
            build_cli()
        return OUT
    BUILD.mkdir(exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    link = [_nvcc(), *ARCH, "-shared", "-cudart", "shared", "-ccbin", _host_cxx(), "-o", str(OUT) + ".tmp",
            *map(str, objs), "-Xlinker", f"-rpath,{cuda}/lib64", "-lpthread"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(str(OUT) + ".tmp", OUT)
    build_cli()
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
