"""The terawarp command (the TeraWarp command line, README.md:85-100;
plugin_Bigimagewarp.cpp:73-107): argument handling on the CPU, and on the GPU
the same files as the library's tw_bigimagewarp_files, byte for byte."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "terawarp_b200" / "terawarp"


@pytest.fixture(scope="module", autouse=True)
def built():
    from terawarp_b200 import build
    build.build()
    assert CLI.exists()


def run(*args):
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, timeout=600)


def test_help_and_argument_errors():
    r = run("--help")
    assert r.returncode == 0 and "usage: terawarp" in r.stdout
    assert run().returncode == 2                                            # no paths
    assert run("-i", "a", "b", "-o", "d", "-p", "1", "1", "0").returncode == 2  # two inputs
    r = run("-i", "a", "b", "c", "-o", "d", "-p", "1", "1", "0", "0", "0")     # five -p values
    assert r.returncode == 2 and "-p takes" in r.stderr
    assert run("-i", "a", "b", "c", "-o", "d", "-p", "2", "1", "0").returncode == 2  # program_mode
    assert run("-i", "a", "b", "c", "-o", "d", "-p", "1", "x", "0").returncode == 2
    assert run("-i", "a", "b", "c", "-o", "d", "-p", "1", "1", "0", "--interp", "cubic").returncode == 2


def test_missing_inputs_fail_with_the_library_message(tmp_path):
    # with a GPU: the marker file is missing; without one: no context
    r = run("-i", tmp_path / "none.v3draw", tmp_path / "s.marker", tmp_path / "t.marker", "-o", tmp_path,
            "-p", "1", "1", "0", "0", "0", "0", "0")
    assert r.returncode == 1 and r.stderr.startswith("terawarp:")


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["plugin", "readme"])
def test_cli_equals_library_call(ctx, tmp_path, form):
    from terawarp_b200 import api, synth
    c = synth.large_tps_case(seed=33, device="cpu", shape_zyx=(40, 70, 90), n=30, g=8, n_blobs=60, n_fibres=8)
    vol = c.vol.numpy()
    api.write_markers(tmp_path / "sub.marker", c.marker_sub)
    api.write_markers(tmp_path / "tar.marker", c.marker_tar)
    api.v3draw_write(tmp_path / "brain.v3draw", vol)
    a, b = tmp_path / "cli", tmp_path / "lib"
    os.makedirs(a)
    os.makedirs(b)
    if form == "plugin":
        p = ["1", "1", "1", "0", "0", "0", "0"]            # TPS, GPU, downsample
        kw = dict(warp_mode=0, deformation_mode=1, downsample_mode=1)
        names = ["brain_stps.v3draw", "brain_stps_downsample.v3draw"]
    else:
        p = ["1", "1", "0", "0", "10", "-5", "20", "0", "0", "0"]   # rigid rotation
        kw = dict(warp_mode=1, deformation_mode=0, para=(10.0, -5.0, 20.0))
        names = None
    r = run("-i", tmp_path / "brain.v3draw", tmp_path / "sub.marker", tmp_path / "tar.marker", "-o", a, "-p", *p)
    assert r.returncode == 0, r.stderr
    api.bigimagewarp_files(ctx, str(tmp_path / "brain.v3draw"), str(tmp_path / "sub.marker"),
                           str(tmp_path / "tar.marker"), str(b), **kw)
    got = sorted(os.listdir(a))
    assert got == sorted(os.listdir(b)) and got
    if names:
        assert set(names) <= set(got)
    for n in got:
        assert (a / n).read_bytes() == (b / n).read_bytes(), n
