"""ctypes binding of the FP64 CPU oracle (oracle/tw_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker; the product path never imports
it.  Parity status: unpinned (the reference has no golden vectors and cannot
be built here); see tw_oracle.c's header.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libtw_oracle.so"
_lib = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build() -> Path:
    src = HERE / "tw_oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    lib.or_tps_solve.argtypes = [C.c_int, _f32p, _f32p, C.c_double, C.c_int, _f64p, _f64p]
    lib.or_tps_solve.restype = C.c_int
    lib.or_grid_size.argtypes = [C.c_int64, C.c_int]
    lib.or_grid_size.restype = C.c_int64
    lib.or_tps_grid.argtypes = [C.c_int, _f32p, _f64p, _f64p, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_int64,
                                C.c_int64, C.c_int64, C.c_int, _f32p]
    lib.or_tps_grid.restype = C.c_int
    lib.or_bspline_tb.argtypes = [C.c_int, _f64p]
    lib.or_tps_warp.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_int64, C.c_int64, _f32p, C.c_int64, C.c_int64,
                                C.c_int64, C.c_int, C.c_int, C.c_int, C.c_void_p]
    lib.or_tps_warp.restype = C.c_int
    lib.or_tps_warp_box.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_int64, C.c_int64, _f32p, C.c_int64,
                                    C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int64,
                                    C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_void_p]
    lib.or_tps_warp_box.restype = C.c_int
    lib.or_affine_fit.argtypes = [C.c_int, _f64p, _f64p, _f64p]
    lib.or_affine_fit.restype = C.c_int
    lib.or_affine_warp.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_int64, C.c_int64, _f64p, C.c_int, C.c_int,
                                   C.c_void_p, C.c_int64, C.c_int64, C.c_int64]
    lib.or_affine_warp.restype = C.c_int
    lib.or_downsample_factor.argtypes = [C.c_int64, C.c_int64, C.c_int64]
    lib.or_downsample_factor.restype = C.c_int
    lib.or_max_threads.restype = C.c_int
    _lib = lib
    return lib


def _dt(a: np.ndarray) -> int:
    return {np.dtype(np.uint8): 1, np.dtype(np.uint16): 2}[a.dtype]


def tps_solve(centres, values, lam: float = 0.2, threads: int = 0):
    """(c n x 4, d 4 x 4); centres/values (n, 3) float32 x, y, z."""
    ctr = np.ascontiguousarray(np.asarray(centres, np.float32).reshape(-1, 3))
    val = np.ascontiguousarray(np.asarray(values, np.float32).reshape(-1, 3))
    n = len(ctr)
    c = np.zeros((n, 4), np.float64)
    d = np.zeros((4, 4), np.float64)
    rc = load().or_tps_solve(n, ctr, val, lam, threads, c, d)
    if rc != 0:
        raise RuntimeError(f"oracle tps_solve failed with {rc}")
    return c, d


def grid_size(sz: int, g: int) -> int:
    return int(load().or_grid_size(sz, g))


def tps_grid(centres, c, d, gsz_xyz, g: int, offset=(0, 0, 0), threads: int = 0):
    """Node displacement grid (gz, gy, gx, 3) float32."""
    ctr = np.ascontiguousarray(np.asarray(centres, np.float32).reshape(-1, 3))
    gx, gy, gz = (int(v) for v in gsz_xyz)
    df = np.zeros((gz, gy, gx, 3), np.float32)
    rc = load().or_tps_grid(len(ctr), ctr, np.ascontiguousarray(c, np.float64), np.ascontiguousarray(d, np.float64),
                            gx, gy, gz, g, int(offset[0]), int(offset[1]), int(offset[2]), threads, df)
    if rc != 0:
        raise RuntimeError(f"oracle tps_grid failed with {rc}")
    return df


def tps_warp(src: np.ndarray, df: np.ndarray, g: int, interp: int = 0, threads: int = 0) -> np.ndarray:
    src = np.ascontiguousarray(src)
    Z, Y, X = src.shape
    gz, gy, gx, _ = df.shape
    out = np.zeros_like(src)
    rc = load().or_tps_warp(src.ctypes.data, _dt(src), X, Y, Z, np.ascontiguousarray(df, np.float32), gx, gy, gz, g,
                            interp, threads, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle tps_warp failed with {rc}")
    return out


def tps_warp_box(src: np.ndarray, df: np.ndarray, g: int, box_o_xyz, box_n_xyz, interp: int = 0,
                 threads: int = 0, planes_of: int | None = None) -> np.ndarray:
    """The whole-volume warp's output restricted to the box [o, o + n)
    (x, y, z voxels): an (nz, ny, nx) array equal to that box of tps_warp's
    result.  planes_of = Z says that src holds only the first planes of a
    volume of Z planes (the range rule uses Z); the caller guarantees that the
    box's samples read no plane beyond those given."""
    src = np.ascontiguousarray(src)
    Z, Y, X = src.shape
    if planes_of is not None:
        if planes_of < Z:
            raise ValueError("planes_of must be at least the planes given")
        Z = int(planes_of)
    gz, gy, gx, _ = df.shape
    ox, oy, oz = (int(v) for v in box_o_xyz)
    nx, ny, nz = (int(v) for v in box_n_xyz)
    out = np.zeros((nz, ny, nx), src.dtype)
    rc = load().or_tps_warp_box(src.ctypes.data, _dt(src), X, Y, Z, np.ascontiguousarray(df, np.float32), gx, gy,
                                gz, g, interp, threads, ox, oy, oz, nx, ny, nz, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle tps_warp_box failed with {rc}")
    return out


def imgwarp_smallmemory_image(ql_marker_tar, ql_marker_sub, g: int, img: np.ndarray, interp_img: int = 0,
                              threads: int = 0, lam: float = 0.2):
    """Whole pipeline of imgwarp_smallmemory_image (q_imgwarp_tps_quicksmallmemory.cpp:1997-2162):
    centres = ql_marker_sub, values = ql_marker_tar."""
    Z, Y, X = img.shape
    c, d = tps_solve(ql_marker_sub, ql_marker_tar, lam, threads)
    gsz = (grid_size(X, g), grid_size(Y, g), grid_size(Z, g))
    df = tps_grid(ql_marker_sub, c, d, gsz, g, threads=threads)
    return tps_warp(img, df, g, interp_img, threads)


def affine_fit(tar, sub) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(tar, np.float64).reshape(-1, 3))
    b = np.ascontiguousarray(np.asarray(sub, np.float64).reshape(-1, 3))
    M = np.zeros(16, np.float64)
    rc = load().or_affine_fit(len(a), a, b, M)
    if rc != 0:
        raise RuntimeError(f"oracle affine_fit failed with {rc}")
    return M.reshape(4, 4)


def affine_warp(src: np.ndarray, M, out_shape_zyx=None, interp: int = 0, threads: int = 0) -> np.ndarray:
    src = np.ascontiguousarray(src)
    Z, Y, X = src.shape
    oz, oy, ox = out_shape_zyx or src.shape
    out = np.zeros((oz, oy, ox), src.dtype)
    rc = load().or_affine_warp(src.ctypes.data, _dt(src), X, Y, Z, np.ascontiguousarray(np.asarray(M, np.float64).reshape(16)),
                               interp, threads, out.ctypes.data, ox, oy, oz)
    if rc != 0:
        raise RuntimeError(f"oracle affine_warp failed with {rc}")
    return out


def downsample_factor(sz_xyz) -> int:
    return int(load().or_downsample_factor(*[int(v) for v in sz_xyz]))


def max_threads() -> int:
    return int(load().or_max_threads())
