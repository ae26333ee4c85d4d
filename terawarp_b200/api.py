"""Python mirror of the TeraWarp warp operators over the C ABI.

Names, argument order and meaning follow the reference's operator functions
(q_imgwarp_tps_quicksmallmemory.h:70-74, q_warp_affine_tps.h:66-74) and the
plugin's parameter surface (plugin_Bigimagewarp.cpp:123-336, README.md:85-100);
volumes are arrays instead of files.  Every call goes through
libterawarp_b200.so; nothing here computes a warp in Python.

Volumes are numpy arrays or torch tensors (host, pinned host or CUDA), C
contiguous, shaped (z, y, x) or (c, z, y, x), dtype uint8 or uint16 -- the
reference's x-fastest layout (basic_memory.cpp:148-168).  Landmarks are (n, 3)
arrays of x, y, z voxel coordinates.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib as L


class TeraWarpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


def _check(status: int, ctx: Optional["Context"] = None, what: str = "") -> None:
    if status == L.TW_OK:
        return
    lib = L.load()
    detail = ""
    if ctx is not None and ctx.handle:
        detail = (lib.tw_ctx_last_error(ctx.handle) or b"").decode()
    base = (lib.tw_status_string(status) or b"").decode()
    raise TeraWarpError(status, f"{what}: {base}" + (f": {detail}" if detail else ""))


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x) -> int:
    if _is_torch(x):
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        if not x.flags.c_contiguous:
            raise ValueError("array must be C contiguous")
        return x.ctypes.data
    raise TypeError(f"unsupported buffer type {type(x)}")


def _stream_arg(stream, *bufs) -> int:
    """The stream handle for a device call.  With no stream the library runs
    the call on the context's own stream and returns when it is complete;
    work that torch has queued on its current stream for these tensors
    (their producers) is finished first, since the context's stream is not
    ordered after torch's."""
    if stream:
        return int(stream)
    import torch
    for b in bufs:
        if _is_torch(b) and b.is_cuda:
            torch.cuda.current_stream(b.device).synchronize()
            break
    return 0


def _dtype_code(x) -> int:
    if _is_torch(x):
        import torch
        if x.dtype == torch.uint8:
            return L.TW_U8
        if x.dtype == torch.uint16:
            return L.TW_U16
        raise TypeError(f"unsupported dtype {x.dtype}")
    if x.dtype == np.uint8:
        return L.TW_U8
    if x.dtype == np.uint16:
        return L.TW_U16
    raise TypeError(f"unsupported dtype {x.dtype}")


def _sz4(x) -> "C.Array":
    shp = tuple(x.shape)
    if len(shp) == 3:
        z, y, xx = shp
        c = 1
    elif len(shp) == 4:
        c, z, y, xx = shp
    else:
        raise ValueError("volume must be (z, y, x) or (c, z, y, x)")
    return (C.c_int64 * 4)(xx, y, z, c)


def _sz3(x) -> "C.Array":
    s = _sz4(x)
    return (C.c_int64 * 3)(s[0], s[1], s[2])


def _pair_count(a, b, what: str) -> int:
    """Number of landmark pairs of two (n, 3) point sets; the C side reads n
    points from both arrays, so a shorter second set would be read past its
    end."""
    na = len(np.asarray(a, dtype=np.float64).reshape(-1, 3))
    nb = len(np.asarray(b, dtype=np.float64).reshape(-1, 3))
    if na != nb:
        raise ValueError(f"{what}: the two landmark sets differ in length ({na} vs {nb})")
    return na


def _markers(pts) -> "C.Array":
    a = np.ascontiguousarray(np.asarray(pts, dtype=np.float32).reshape(-1, 3))
    if len(a) == 0:
        return (L.tw_marker * 1)()
    # tw_marker is three packed floats, the same bytes as an (n, 3) float32 array
    return (L.tw_marker * len(a)).from_buffer_copy(a.tobytes())


def _like(x, shape):
    if _is_torch(x):
        import torch
        kw = {"dtype": x.dtype, "device": x.device}
        if x.device.type == "cpu" and x.is_pinned():
            return torch.empty(shape, pin_memory=True, dtype=x.dtype)
        return torch.empty(shape, **kw)
    return np.empty(shape, dtype=x.dtype)


class Context:
    """A device context (tw_ctx): streams, HBM budget, error text."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.lib = L.load()
        h = C.c_void_p()
        _check(self.lib.tw_ctx_create(device, hbm_budget_bytes, C.byref(h)), None, "tw_ctx_create")
        self.handle = h
        self.device = device

    def close(self) -> None:
        if self.handle:
            self.lib.tw_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.tw_ctx_kernel_launches(self.handle))

    @property
    def transfer_bytes(self):
        """(host -> device, device -> host) bytes the streaming paths moved."""
        a, b = C.c_uint64(), C.c_uint64()
        self.lib.tw_ctx_transfer_bytes(self.handle, C.byref(a), C.byref(b))
        return int(a.value), int(b.value)

    def synchronize(self) -> None:
        _check(self.lib.tw_ctx_synchronize(self.handle), self, "tw_ctx_synchronize")


class TPS:
    """Solved TPS coefficients, device-resident (tw_tps)."""

    def __init__(self, ctx: Context, handle: C.c_void_p, n: int):
        self.ctx, self.handle, self.n = ctx, handle, n

    def coeffs(self):
        c = np.zeros((self.n, 4), np.float64)
        d = np.zeros((4, 4), np.float64)
        _check(self.ctx.lib.tw_tps_get_coeffs(self.handle, c.ctypes.data_as(L._DP), d.ctypes.data_as(L._DP)),
               self.ctx, "tw_tps_get_coeffs")
        return c, d

    def close(self) -> None:
        if self.handle:
            self.ctx.lib.tw_tps_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tps_solve(ctx: Context, centres, values, lam: float = 0.2) -> TPS:
    """FP64 GPU solve; centres = TPS kernel centres, values = mapped points."""
    n = _pair_count(centres, values, "tps_solve")
    c = _markers(centres)
    v = _markers(values)
    h = C.c_void_p()
    _check(ctx.lib.tw_tps_solve(ctx.handle, c, v, n, lam, C.byref(h)), ctx, "tw_tps_solve")
    return TPS(ctx, h, n)


def grid_size(sz: int, g: int) -> int:
    return int(L.load().tw_grid_size(sz, g))


def tps_eval_grid(ctx: Context, tps: TPS, gsz: Sequence[int], g: int, offset=(0, 0, 0), out=None, stream=None):
    """Node displacements (gz, gy, gx, 4) float32 on the context's device."""
    import torch
    gx, gy, gz = (int(v) for v in gsz)
    if out is None:
        out = torch.empty((gz, gy, gx, 4), dtype=torch.float32, device=f"cuda:{ctx.device}")
    _check(ctx.lib.tw_tps_eval_grid(ctx.handle, tps.handle, gx, gy, gz, g, int(offset[0]), int(offset[1]),
                                    int(offset[2]), C.c_void_p(_ptr(out)), C.c_void_p(_stream_arg(stream, out))),
           ctx, "tw_tps_eval_grid")
    return out


def warp_tps_device(ctx: Context, nodes, g: int, src, dst, interp: int = 0, stream=None) -> None:
    """Fused B-spline + resample of device volumes (z, y, x)."""
    _check(ctx.lib.tw_warp_tps_device(ctx.handle, C.c_void_p(_ptr(nodes)), g, _dtype_code(src), interp,
                                      C.c_void_p(_ptr(src)), C.c_void_p(_ptr(dst)), _sz3(src),
                                      C.c_void_p(_stream_arg(stream, nodes, src, dst))), ctx, "tw_warp_tps_device")


def fit_affine(ctx: Context, tar, sub) -> np.ndarray:
    """4x4 matrix T with sub = T tar (3-D DLT, FP64 on the GPU)."""
    M = np.zeros(16, np.float64)
    n = _pair_count(tar, sub, "fit_affine")
    _check(ctx.lib.tw_fit_affine(ctx.handle, _markers(tar), _markers(sub), n, M.ctypes.data_as(L._DP)), ctx,
           "tw_fit_affine")
    return M.reshape(4, 4)


FIT_AFFINE_NOALLOC_MAX = 4096


def fit_affine_noalloc(ctx: Context, tar, sub) -> np.ndarray:
    """fit_affine through tw_fit_affine_noalloc: same result, no allocation;
    at most FIT_AFFINE_NOALLOC_MAX landmark pairs."""
    M = np.zeros(16, np.float64)
    n = _pair_count(tar, sub, "fit_affine_noalloc")
    _check(ctx.lib.tw_fit_affine_noalloc(ctx.handle, _markers(tar), _markers(sub), n, M.ctypes.data_as(L._DP)),
           ctx, "tw_fit_affine_noalloc")
    return M.reshape(4, 4)


def make_affine(warp_mode: int, deformation_mode: int, para, in_sz, out_sz=None) -> np.ndarray:
    """Pull-back matrix of the scaling / rotation / translation parameters."""
    out_sz = in_sz if out_sz is None else out_sz
    M = np.zeros(16, np.float64)
    p = (C.c_double * 3)(*[float(v) for v in para])
    a = (C.c_int64 * 3)(*[int(v) for v in in_sz])
    b = (C.c_int64 * 3)(*[int(v) for v in out_sz])
    _check(L.load().tw_make_affine(warp_mode, deformation_mode, p, a, b, M.ctypes.data_as(L._DP)), None,
           "tw_make_affine")
    return M.reshape(4, 4)


def warp_affine_device(ctx: Context, M, src, dst, interp: int = 0, stream=None) -> None:
    Mx = np.ascontiguousarray(np.asarray(M, np.float64).reshape(16))
    _check(ctx.lib.tw_warp_affine_device(ctx.handle, Mx.ctypes.data_as(L._DP), _dtype_code(src), interp,
                                         C.c_void_p(_ptr(src)), _sz3(src), C.c_void_p(_ptr(dst)), _sz3(dst),
                                         C.c_void_p(_stream_arg(stream, src, dst))), ctx, "tw_warp_affine_device")


def imgwarp_smallmemory_image(ctx: Context, ql_marker_tar, ql_marker_sub, szBlock_x: int, szBlock_y: int,
                              szBlock_z: int, i_interpmethod_df: int, i_interpmethod_img: int, p_img_sub, out=None):
    """Mirror of imgwarp_smallmemory_image: ql_marker_tar are the TPS values,
    ql_marker_sub the TPS centres (as the reference function uses them)."""
    if out is None:
        out = _like(p_img_sub, tuple(p_img_sub.shape))
    n = len(np.asarray(ql_marker_tar).reshape(-1, 3))
    if len(np.asarray(ql_marker_sub).reshape(-1, 3)) != n:
        raise TeraWarpError(L.TW_ERR_ARG, "target or subject control points is invalid")
    _check(ctx.lib.tw_imgwarp_smallmemory_image(ctx.handle, _markers(ql_marker_tar), _markers(ql_marker_sub), n,
                                                szBlock_x, szBlock_y, szBlock_z, i_interpmethod_df,
                                                i_interpmethod_img, _dtype_code(p_img_sub),
                                                C.c_void_p(_ptr(p_img_sub)), _sz4(p_img_sub),
                                                C.c_void_p(_ptr(out))), ctx, "imgwarp_smallmemory_image")
    return out


def q_imagewarp_affine_image(ctx: Context, ql_marker_tar, ql_marker_sub, p_img_sub, out=None):
    """Mirror of q_imagewarp_affine_image: fits sub = T tar and warps."""
    if out is None:
        out = _like(p_img_sub, tuple(p_img_sub.shape))
    n = len(np.asarray(ql_marker_tar).reshape(-1, 3))
    if len(np.asarray(ql_marker_sub).reshape(-1, 3)) != n:
        raise TeraWarpError(L.TW_ERR_ARG, "target or subject control points is invalid")
    _check(ctx.lib.tw_q_imagewarp_affine_image(ctx.handle, _markers(ql_marker_tar), _markers(ql_marker_sub), n,
                                               _dtype_code(p_img_sub), C.c_void_p(_ptr(p_img_sub)), _sz4(p_img_sub),
                                               C.c_void_p(_ptr(out))), ctx, "q_imagewarp_affine_image")
    return out


def _tile_opts(tile, depth, interp, region=None) -> L.tw_tile_opts:
    o = L.tw_tile_opts()
    for a in range(3):
        o.tile[a] = int(tile[a]) if tile is not None else 0
    o.staging_depth = int(depth)
    o.interp = int(interp)
    if region is not None:
        (ox, oy, oz), (nx, ny, nz) = region
        for a, (ov, nv) in enumerate(((ox, nx), (oy, ny), (oz, nz))):
            o.region_o[a] = int(ov)
            o.region_n[a] = int(nv)
    return o


class SyntheticVolume:
    """A procedural tile source (tw_synthetic_volume): voxels from a seeded
    hash of their coordinates, no storage; shape (z, y, x)."""

    def __init__(self, shape_zyx, dtype, seed: int = 1, threads: int = 0):
        self.v = L.tw_synthetic_volume()
        self.v.seed = int(seed)
        self.v.sz[0], self.v.sz[1], self.v.sz[2] = int(shape_zyx[2]), int(shape_zyx[1]), int(shape_zyx[0])
        self.dtype_code = L.TW_U8 if np.dtype(dtype) == np.uint8 else L.TW_U16
        self.v.dtype = self.dtype_code
        self.v.threads = int(threads)
        self.shape = tuple(int(s) for s in shape_zyx)
        self.shape_xyz = (self.shape[2], self.shape[1], self.shape[0])
        self.dtype = np.dtype(dtype)
        self.handle = C.cast(C.pointer(self.v), C.c_void_p)

    def read_box(self, o_xyz, n_xyz) -> np.ndarray:
        nx, ny, nz = (int(v) for v in n_xyz)
        a = np.empty((nz, ny, nx), self.dtype)
        rc = L.load().tw_box_reader_synthetic(self.handle, int(o_xyz[0]), int(o_xyz[1]), int(o_xyz[2]), nx, ny, nz,
                                              a.ctypes.data)
        if rc != 0:
            raise TeraWarpError(L.TW_ERR_IO, f"synthetic read failed ({rc})")
        return a


class Checksum:
    """A sink that keeps the sum, a position-weighted sum and the voxel count
    of what it receives (tw_checksum)."""

    def __init__(self, dtype, threads: int = 0):
        self.c = L.tw_checksum()
        self.c.dtype = L.TW_U8 if np.dtype(dtype) == np.uint8 else L.TW_U16
        self.c.threads = int(threads)
        self.handle = C.cast(C.pointer(self.c), C.c_void_p)

    def write_box(self, o_xyz, block) -> None:
        b = np.ascontiguousarray(block)
        nz, ny, nx = b.shape
        L.load().tw_box_writer_checksum(self.handle, int(o_xyz[0]), int(o_xyz[1]), int(o_xyz[2]), nx, ny, nz,
                                        b.ctypes.data)

    @property
    def value(self):
        return int(self.c.sum), int(self.c.weighted), int(self.c.voxels)


def _host_volume(x) -> L.tw_host_volume:
    if _is_torch(x) and x.is_cuda:
        raise ValueError("tiled paths stream host volumes; pass a host array")
    v = L.tw_host_volume()
    v.data = _ptr(x)
    s = _sz3(x)
    for a in range(3):
        v.sz[a] = s[a]
    v.dtype = _dtype_code(x)
    v.threads = 0
    return v


def _box_io(src, dst, read_fn=None, write_fn=None):
    """Tile source / sink: the library's built-in host-volume reader and writer
    (strided DMA when the array is pinned), a SliceDir / SliceWriter, or
    Python callables read_fn(x0, y0, z0, nx, ny, nz) -> array(nz, ny, nx) and
    write_fn(x0, y0, z0, block) for testing the callback path."""
    lib = L.load()
    keep = []
    if isinstance(src, SliceDir):
        rd = L.READ_BOX(C.cast(lib.tw_box_reader_slices, C.c_void_p).value)
        ru = src.handle
    elif isinstance(src, SyntheticVolume):
        rd = L.READ_BOX(C.cast(lib.tw_box_reader_synthetic, C.c_void_p).value)
        ru = src.handle
    elif read_fn is None:
        hv_in = _host_volume(src)
        keep.append(hv_in)
        rd = L.READ_BOX(C.cast(lib.tw_box_reader_host, C.c_void_p).value)
        ru = C.cast(C.pointer(hv_in), C.c_void_p)
    else:
        es = 1 if _src_dtype(src) == L.TW_U8 else 2

        def _rd(user, x0, y0, z0, nx, ny, nz, dstp):
            try:
                blk = np.ascontiguousarray(read_fn(x0, y0, z0, nx, ny, nz))
                C.memmove(dstp, blk.ctypes.data, nx * ny * nz * es)
                return 0
            except Exception:
                return 1
        rd = L.READ_BOX(_rd)
        ru = None
    if isinstance(dst, SliceWriter):
        wr = L.WRITE_BOX(C.cast(lib.tw_box_writer_slices, C.c_void_p).value)
        wu = dst.handle
    elif isinstance(dst, Checksum):
        wr = L.WRITE_BOX(C.cast(lib.tw_box_writer_checksum, C.c_void_p).value)
        wu = dst.handle
    elif write_fn is None:
        hv_out = _host_volume(dst)
        keep.append(hv_out)
        wr = L.WRITE_BOX(C.cast(lib.tw_box_writer_host, C.c_void_p).value)
        wu = C.cast(C.pointer(hv_out), C.c_void_p)
    else:
        dt = np.uint8 if _src_dtype(src) == L.TW_U8 else np.uint16

        def _wr(user, x0, y0, z0, nx, ny, nz, srcp):
            try:
                buf = (C.c_char * (nx * ny * nz * np.dtype(dt).itemsize)).from_address(srcp)
                write_fn(x0, y0, z0, np.frombuffer(buf, dtype=dt).reshape(nz, ny, nx).copy())
                return 0
            except Exception:
                return 1
        wr = L.WRITE_BOX(_wr)
        wu = None
    keep += [rd, wr]
    return rd, ru, wr, wu, keep


def _src_dtype(src) -> int:
    return src.dtype_code if isinstance(src, (SliceDir, SyntheticVolume)) else _dtype_code(src)


def _src_sz3(src):
    if isinstance(src, (SliceDir, SyntheticVolume)):
        return (C.c_int64 * 3)(*src.shape_xyz)
    return _sz3(src)


def imgwarp_smallmemory_tiled(ctx: Context, ql_marker_tar, ql_marker_sub, marker_scale: float, g: int, src, out=None,
                              tile=(512, 512, 512), depth: int = 2, interp: int = 0, read_fn=None, write_fn=None,
                              region=None):
    """Mirror of imgwarp_smallmemory_CYF for volumes streamed tile by tile
    (the source may exceed HBM): centres = ql_marker_sub, values =
    ql_marker_tar, both scaled by marker_scale.  src: a host array, a
    SliceDir or a SyntheticVolume; out: a host array, a SliceWriter or a
    Checksum.  region: ((x0, y0, z0), (nx, ny, nz)) of the output to warp."""
    if out is None and write_fn is None:
        out = _like(src, tuple(src.shape))
    n = _pair_count(ql_marker_tar, ql_marker_sub, "imgwarp_smallmemory_tiled")
    rd, ru, wr, wu, keep = _box_io(src, out, read_fn, write_fn)
    opts = _tile_opts(tile, depth, interp, region)
    _check(ctx.lib.tw_imgwarp_smallmemory_tiled(ctx.handle, _markers(ql_marker_tar), _markers(ql_marker_sub), n,
                                                marker_scale, g, _src_dtype(src), _src_sz3(src), rd, ru, wr, wu,
                                                C.byref(opts)), ctx, "tw_imgwarp_smallmemory_tiled")
    del keep
    return out


def warp_affine_tiled(ctx: Context, M, src, out_shape_zyx=None, out=None, tile=(512, 512, 512), depth: int = 2,
                      interp: int = 0, read_fn=None, write_fn=None, region=None):
    """Affine warp streamed tile by tile (q_imagewarp_affine_cyf)."""
    shape = tuple(out_shape_zyx) if out_shape_zyx is not None else tuple(src.shape)
    if out is None and write_fn is None:
        out = _like(src, shape)
    Mx = np.ascontiguousarray(np.asarray(M, np.float64).reshape(16))
    rd, ru, wr, wu, keep = _box_io(src, out, read_fn, write_fn)
    opts = _tile_opts(tile, depth, interp, region)
    osz = (C.c_int64 * 3)(shape[2], shape[1], shape[0])
    _check(ctx.lib.tw_warp_affine_tiled(ctx.handle, Mx.ctypes.data_as(L._DP), _src_dtype(src), _src_sz3(src), osz, rd,
                                        ru, wr, wu, C.byref(opts)), ctx, "tw_warp_affine_tiled")
    del keep
    return out


# ------------------------------------------------------------------- files

def _io_check(status: int, what: str) -> None:
    if status != L.TW_OK:
        lib = L.load()
        raise TeraWarpError(status, f"{what}: {(lib.tw_status_string(status) or b'').decode()}")


def v3draw_header(path: str):
    """((x, y, z, channels), dtype code) of a Vaa3D raw stack."""
    sz = (C.c_int64 * 4)()
    dt = C.c_int()
    _io_check(L.load().tw_v3draw_read_header(str(path).encode(), sz, C.byref(dt), None), f"read header {path}")
    return tuple(int(v) for v in sz), int(dt.value)


def v3draw_read(path: str) -> np.ndarray:
    """A raw stack as (z, y, x) (one channel) or (c, z, y, x)."""
    (x, y, z, c), dt = v3draw_header(path)
    npdt = {L.TW_U8: np.uint8, L.TW_U16: np.uint16, 4: np.float32}[dt]
    a = np.empty((c, z, y, x), npdt)
    _io_check(L.load().tw_v3draw_read(str(path).encode(), a.ctypes.data, a.nbytes), f"read {path}")
    return a[0] if c == 1 else a


def v3draw_read_box(path: str, o_xyz, n_xyz) -> np.ndarray:
    """Box [o, o + n) of channel 0 as (nz, ny, nx)."""
    (_, _, _, _), dt = v3draw_header(path)
    npdt = {L.TW_U8: np.uint8, L.TW_U16: np.uint16, 4: np.float32}[dt]
    nx, ny, nz = (int(v) for v in n_xyz)
    a = np.empty((nz, ny, nx), npdt)
    _io_check(L.load().tw_v3draw_read_box(str(path).encode(), int(o_xyz[0]), int(o_xyz[1]), int(o_xyz[2]), nx, ny,
                                          nz, a.ctypes.data), f"read box of {path}")
    return a


def v3draw_write(path: str, arr) -> None:
    a = np.ascontiguousarray(arr)
    _io_check(L.load().tw_v3draw_write(str(path).encode(), a.ctypes.data, _sz4(a), _dtype_code(a)), f"write {path}")


class SliceDir:
    """A directory of per-Z raw slice files as a tile source (tw_slice_dir)."""

    def __init__(self, path: str, threads: int = 0):
        self.lib = L.load()
        h = C.c_void_p()
        _io_check(self.lib.tw_slice_dir_open(str(path).encode(), threads, C.byref(h)), f"open slices {path}")
        self.handle = h
        sz = (C.c_int64 * 3)()
        dt = C.c_int()
        self.lib.tw_slice_dir_info(h, sz, C.byref(dt))
        self.shape_xyz = tuple(int(v) for v in sz)
        self.shape = (self.shape_xyz[2], self.shape_xyz[1], self.shape_xyz[0])
        self.dtype_code = int(dt.value)
        self.dtype = np.uint8 if self.dtype_code == L.TW_U8 else np.uint16

    def read_box(self, o_xyz, n_xyz) -> np.ndarray:
        nx, ny, nz = (int(v) for v in n_xyz)
        a = np.empty((nz, ny, nx), self.dtype)
        rc = self.lib.tw_box_reader_slices(self.handle, int(o_xyz[0]), int(o_xyz[1]), int(o_xyz[2]), nx, ny, nz,
                                           a.ctypes.data)
        if rc != 0:
            raise TeraWarpError(L.TW_ERR_IO, f"slice read failed ({rc})")
        return a

    def close(self) -> None:
        if self.handle:
            self.lib.tw_slice_dir_close(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class SliceWriter:
    """Per-Z raw slice files that output tiles are written into (tw_slice_writer)."""

    def __init__(self, path: str, shape_zyx, dtype, threads: int = 0):
        self.lib = L.load()
        self.dtype_code = L.TW_U8 if np.dtype(dtype) == np.uint8 else L.TW_U16
        sz = (C.c_int64 * 3)(int(shape_zyx[2]), int(shape_zyx[1]), int(shape_zyx[0]))
        h = C.c_void_p()
        _io_check(self.lib.tw_slice_writer_create(str(path).encode(), sz, self.dtype_code, threads, C.byref(h)),
                  f"create slices in {path}")
        self.handle = h
        self.shape = tuple(int(v) for v in shape_zyx)

    def write_box(self, o_xyz, block) -> None:
        b = np.ascontiguousarray(block)
        nz, ny, nx = b.shape
        rc = self.lib.tw_box_writer_slices(self.handle, int(o_xyz[0]), int(o_xyz[1]), int(o_xyz[2]), nx, ny, nz,
                                           b.ctypes.data)
        if rc != 0:
            raise TeraWarpError(L.TW_ERR_IO, f"slice write failed ({rc})")

    def close(self) -> None:
        if self.handle:
            self.lib.tw_slice_writer_close(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def read_slices(path: str) -> np.ndarray:
    """A whole slice directory as one (z, y, x) array."""
    with SliceDir(path) as d:
        x, y, z = d.shape_xyz
        return d.read_box((0, 0, 0), (x, y, z))


def read_markers(path: str) -> np.ndarray:
    """(n, 3) float32 x, y, z of a .marker file."""
    lib = L.load()
    n = C.c_int()
    _io_check(lib.tw_marker_file_read(str(path).encode(), None, 0, C.byref(n)), f"read markers {path}")
    buf = (L.tw_marker * max(1, n.value))()
    _io_check(lib.tw_marker_file_read(str(path).encode(), buf, n.value, C.byref(n)), f"read markers {path}")
    return np.frombuffer(bytes(buf), np.float32).reshape(-1, 3)[:n.value].copy()


def write_markers(path: str, pts) -> None:
    _io_check(L.load().tw_marker_file_write(str(path).encode(), _markers(pts), len(np.asarray(pts).reshape(-1, 3))),
              f"write markers {path}")


def bigimagewarp_files(ctx: Context, img_sub: str, marker_sub: str, marker_tar: str, out_dir: str,
                       downsample_mode: int = 0, **kw) -> None:
    """The plugin's command on files (tw_bigimagewarp_files): a .v3draw file or
    a directory of slices in, <name><suffix>.v3draw or <name><suffix>_slice/
    out (keyword arguments as `params`)."""
    kw.setdefault("marker_scale", 0.0)  # 0: the reference's choice (1 for a .v3draw, 4 for slices)
    p = params(**kw)
    p.downsample_mode = int(downsample_mode)
    _check(ctx.lib.tw_bigimagewarp_files(ctx.handle, C.byref(p), str(img_sub).encode(),
                                         str(marker_sub).encode() if marker_sub else None,
                                         str(marker_tar).encode() if marker_tar else None, str(out_dir).encode()),
           ctx, "tw_bigimagewarp_files")


class Server:
    """Continuous-batching warp server (tw_server): jobs are admitted by HBM
    budget as they arrive, their resample work is batched into persistent
    launches, and results land in the caller's host buffers."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int = 0, max_inflight: int = 16):
        self.ctx = ctx
        h = C.c_void_p()
        _check(ctx.lib.tw_server_create(ctx.handle, hbm_budget_bytes, max_inflight, C.byref(h)), ctx,
               "tw_server_create")
        self.handle = h
        self._keep = {}

    def _submit(self, job: L.tw_job, keep) -> int:
        jid = C.c_uint64()
        _check(self.ctx.lib.tw_server_submit(self.handle, C.byref(job), C.byref(jid)), None, "tw_server_submit")
        self._keep[jid.value] = keep
        return jid.value

    def submit_affine(self, M, src, dst, interp: int = 0) -> int:
        j = L.tw_job()
        j.kind, j.dtype, j.interp, j.g = 0, _dtype_code(src), interp, 0
        s, d = _sz3(src), _sz3(dst)
        for a in range(3):
            j.src_sz[a], j.dst_sz[a] = s[a], d[a]
        for i, v in enumerate(np.asarray(M, np.float64).reshape(16)):
            j.M[i] = float(v)
        j.src, j.dst = _ptr(src), _ptr(dst)
        return self._submit(j, (src, dst))

    def submit_tps(self, centres, values, g: int, src, dst, lam: float = 0.2, interp: int = 0) -> int:
        """centres = target-image landmarks (TPS centres), values = subject-image landmarks."""
        j = L.tw_job()
        j.kind, j.dtype, j.interp, j.g = 1, _dtype_code(src), interp, g
        s, d = _sz3(src), _sz3(dst)
        for a in range(3):
            j.src_sz[a], j.dst_sz[a] = s[a], d[a]
        n = _pair_count(centres, values, "submit_tps")
        c, v = _markers(centres), _markers(values)
        j.centres = C.cast(c, C.POINTER(L.tw_marker))
        j.values = C.cast(v, C.POINTER(L.tw_marker))
        j.n = n
        j.lambda_ = lam
        j.src, j.dst = _ptr(src), _ptr(dst)
        return self._submit(j, (src, dst, c, v))

    def poll(self, job_id: int):
        """(done, latency_s); raises on a failed job."""
        lat = C.c_double()
        st = self.ctx.lib.tw_server_poll(self.handle, job_id, C.byref(lat))
        if st == L.TW_ERR_NOT_READY:
            return False, None
        self._keep.pop(job_id, None)
        _check(st, None, f"server job {job_id}")
        return True, lat.value

    def wait(self, job_id: int, timeout_s: float = 600.0) -> float:
        lat = C.c_double()
        st = self.ctx.lib.tw_server_wait(self.handle, job_id, timeout_s, C.byref(lat))
        self._keep.pop(job_id, None)
        _check(st, None, f"server job {job_id}")
        return lat.value

    def job_times(self, job_id: int) -> dict:
        """Stage times (seconds) of a finished job: queue wait before
        admission, then solve / node grid / inputs resident / resample start /
        resample end / result in place measured from admission on the GPU
        clock (None where a stage does not apply), and the total latency."""
        t = np.zeros(8, np.float64)
        _check(self.ctx.lib.tw_server_job_times(self.handle, job_id, t.ctypes.data_as(L._DP)), None,
               f"server job {job_id} times")
        names = ["queued", "solve", "grid", "ready", "resample_start", "resample_end", "done", "latency"]
        return {k: (None if v < 0 else float(v)) for k, v in zip(names, t)}

    def close(self) -> None:
        if self.handle:
            self.ctx.lib.tw_server_destroy(self.handle)
            self.handle = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def params(warp_mode=0, device_mode=1, resize_mode=0, deformation_mode=1, para=(1.0, 1.0, 1.0), newsize=(0, 0, 0),
           grid_spacing=4, marker_scale=1.0, lam=0.2, interp=0) -> L.tw_params:
    p = L.tw_params()
    L.load().tw_params_default(C.byref(p))
    p.warp_mode, p.device_mode, p.resize_mode, p.deformation_mode = warp_mode, device_mode, resize_mode, \
        deformation_mode
    p.para_x, p.para_y, p.para_z = (float(v) for v in para)
    p.newsize_x, p.newsize_y, p.newsize_z = (int(v) for v in newsize)
    p.grid_spacing, p.marker_scale, p.lambda_, p.interp = grid_spacing, marker_scale, lam, interp
    return p


def output_size(p: L.tw_params, in_sz) -> tuple:
    a = (C.c_int64 * 3)(*[int(v) for v in in_sz])
    b = (C.c_int64 * 3)()
    _check(L.load().tw_output_size(C.byref(p), a, b), None, "tw_output_size")
    return tuple(int(v) for v in b)


def bigimagewarp(ctx: Context, p_img_sub, marker_sub=None, marker_tar=None, out=None, **kw):
    """Plugin-level warp with the TeraWarp command's parameters (keyword
    arguments of `params`)."""
    p = params(**kw)
    sz4 = _sz4(p_img_sub)
    osz = output_size(p, (sz4[0], sz4[1], sz4[2]))
    shape = (osz[2], osz[1], osz[0]) if len(p_img_sub.shape) == 3 else (sz4[3], osz[2], osz[1], osz[0])
    if out is None:
        out = _like(p_img_sub, shape)
    n = 0 if marker_sub is None else _pair_count(marker_sub, marker_tar, "bigimagewarp")
    ms = _markers(marker_sub if marker_sub is not None else np.zeros((1, 3)))
    mt = _markers(marker_tar if marker_tar is not None else np.zeros((1, 3)))
    _check(ctx.lib.tw_bigimagewarp(ctx.handle, C.byref(p), ms, mt, n, _dtype_code(p_img_sub),
                                   C.c_void_p(_ptr(p_img_sub)), sz4, C.c_void_p(_ptr(out))), ctx, "tw_bigimagewarp")
    return out


def downsample_factor(sz) -> int:
    a = (C.c_int64 * 3)(*[int(v) for v in sz])
    return int(L.load().tw_downsample_factor(a))


def downsample_image(ctx: Context, img, out=None):
    sz4 = _sz4(img)
    f = downsample_factor((sz4[0], sz4[1], sz4[2]))
    osz = (sz4[0] // f, sz4[1] // f, sz4[2] // f)
    shape = (osz[2], osz[1], osz[0]) if len(img.shape) == 3 else (sz4[3], osz[2], osz[1], osz[0])
    if out is None:
        out = _like(img, shape)
    o3 = (C.c_int64 * 3)()
    _check(ctx.lib.tw_downsample_image(ctx.handle, _dtype_code(img), C.c_void_p(_ptr(img)), sz4,
                                       C.c_void_p(_ptr(out)), o3), ctx, "tw_downsample_image")
    return out
