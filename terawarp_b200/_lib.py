"""ctypes binding of libterawarp_b200.so (the C ABI in include/terawarp_b200.h).

The shared library is the product; this module only declares its signatures.
Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libterawarp_b200.so"

TW_OK, TW_ERR_ARG, TW_ERR_SINGULAR, TW_ERR_OOM, TW_ERR_CUDA, TW_ERR_TIMEOUT, TW_ERR_IO, TW_ERR_UNSUPPORTED, \
    TW_ERR_NOT_READY = range(9)
TW_U8, TW_U16 = 1, 2


class tw_marker(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class tw_host_volume(C.Structure):
    _fields_ = [("data", C.c_void_p), ("sz", C.c_int64 * 3), ("dtype", C.c_int), ("threads", C.c_int)]


class tw_synthetic_volume(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("sz", C.c_int64 * 3), ("dtype", C.c_int), ("threads", C.c_int)]


class tw_checksum(C.Structure):
    _fields_ = [("sum", C.c_uint64), ("weighted", C.c_uint64), ("voxels", C.c_uint64), ("dtype", C.c_int),
                ("threads", C.c_int)]


class tw_tile_opts(C.Structure):
    _fields_ = [("tile", C.c_int64 * 3), ("staging_depth", C.c_int), ("interp", C.c_int),
                ("region_o", C.c_int64 * 3), ("region_n", C.c_int64 * 3)]


class tw_tile_candidate(C.Structure):
    _fields_ = [("tile", C.c_int64 * 3), ("staging_depth", C.c_int), ("seconds", C.c_double)]


class tw_params(C.Structure):
    _fields_ = [
        ("warp_mode", C.c_int), ("device_mode", C.c_int), ("resize_mode", C.c_int), ("deformation_mode", C.c_int),
        ("para_x", C.c_double), ("para_y", C.c_double), ("para_z", C.c_double),
        ("newsize_x", C.c_int64), ("newsize_y", C.c_int64), ("newsize_z", C.c_int64),
        ("grid_spacing", C.c_int), ("marker_scale", C.c_double), ("lambda_", C.c_double), ("interp", C.c_int),
        ("downsample_mode", C.c_int),
    ]


class tw_job(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("dtype", C.c_int), ("interp", C.c_int), ("g", C.c_int),
        ("src_sz", C.c_int64 * 3), ("dst_sz", C.c_int64 * 3), ("M", C.c_double * 16),
        ("centres", C.POINTER(tw_marker)), ("values", C.POINTER(tw_marker)), ("n", C.c_int),
        ("lambda_", C.c_double), ("src", C.c_void_p), ("dst", C.c_void_p),
    ]


READ_BOX = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                       C.c_void_p)
WRITE_BOX = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                        C.c_void_p)

_P = C.c_void_p
_I64P = C.POINTER(C.c_int64)
_DP = C.POINTER(C.c_double)
_MP = C.POINTER(tw_marker)

# name -> (restype, argtypes); every function the header declares
SIGNATURES = {
    "tw_ctx_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(_P)]),
    "tw_ctx_destroy": (C.c_int, [_P]),
    "tw_ctx_last_error": (C.c_char_p, [_P]),
    "tw_status_string": (C.c_char_p, [C.c_int]),
    "tw_abi_version": (C.c_int, []),
    "tw_ctx_kernel_launches": (C.c_uint64, [_P]),
    "tw_ctx_transfer_bytes": (None, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "tw_ctx_synchronize": (C.c_int, [_P]),
    "tw_tps_solve": (C.c_int, [_P, _MP, _MP, C.c_int, C.c_double, C.POINTER(_P)]),
    "tw_tps_destroy": (C.c_int, [_P]),
    "tw_tps_count": (C.c_int, [_P]),
    "tw_tps_get_coeffs": (C.c_int, [_P, _DP, _DP]),
    "tw_tps_eval_grid": (C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_int64, C.c_int64,
                                   C.c_int64, _P, _P]),
    "tw_grid_size": (C.c_int64, [C.c_int64, C.c_int]),
    "tw_warp_tps_device": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _P, _P, _I64P, _P]),
    "tw_fit_affine": (C.c_int, [_P, _MP, _MP, C.c_int, _DP]),
    "tw_fit_affine_noalloc": (C.c_int, [_P, _MP, _MP, C.c_int, _DP]),
    "tw_make_affine": (C.c_int, [C.c_int, C.c_int, _DP, _I64P, _I64P, _DP]),
    "tw_warp_affine_device": (C.c_int, [_P, _DP, C.c_int, C.c_int, _P, _I64P, _P, _I64P, _P]),
    "tw_imgwarp_smallmemory_image": (C.c_int, [_P, _MP, _MP, C.c_int, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                                               C.c_int, C.c_int, _P, _I64P, _P]),
    "tw_q_imagewarp_affine_image": (C.c_int, [_P, _MP, _MP, C.c_int, C.c_int, _P, _I64P, _P]),
    "tw_imgwarp_smallmemory_tiled": (C.c_int, [_P, _MP, _MP, C.c_int, C.c_double, C.c_int, C.c_int, _I64P,
                                               READ_BOX, _P, WRITE_BOX, _P, C.POINTER(tw_tile_opts)]),
    "tw_warp_affine_tiled": (C.c_int, [_P, _DP, C.c_int, _I64P, _I64P, READ_BOX, _P, WRITE_BOX, _P,
                                       C.POINTER(tw_tile_opts)]),
    "tw_tune_tiled_tps": (C.c_int, [_P, _MP, _MP, C.c_int, C.c_double, C.c_int, C.c_int, _I64P, READ_BOX, _P,
                                    C.POINTER(tw_tile_candidate), C.c_int, _I64P, C.c_char_p,
                                    C.POINTER(tw_tile_opts)]),
    "tw_box_reader_host": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _P]),
    "tw_box_writer_host": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _P]),
    "tw_params_default": (None, [C.POINTER(tw_params)]),
    "tw_output_size": (C.c_int, [C.POINTER(tw_params), _I64P, _I64P]),
    "tw_bigimagewarp": (C.c_int, [_P, C.POINTER(tw_params), _MP, _MP, C.c_int, C.c_int, _P, _I64P, _P]),
    "tw_downsample_factor": (C.c_int, [_I64P]),
    "tw_downsample_image": (C.c_int, [_P, C.c_int, _P, _I64P, _P, _I64P]),
    "tw_box_reader_synthetic": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                          _P]),
    "tw_box_writer_checksum": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _P]),
    "tw_v3draw_read_header": (C.c_int, [C.c_char_p, _I64P, C.POINTER(C.c_int), _I64P]),
    "tw_v3draw_read": (C.c_int, [C.c_char_p, _P, C.c_size_t]),
    "tw_v3draw_read_box": (C.c_int, [C.c_char_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                     _P]),
    "tw_v3draw_write": (C.c_int, [C.c_char_p, _P, _I64P, C.c_int]),
    "tw_slice_dir_open": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(_P)]),
    "tw_slice_dir_info": (C.c_int, [_P, _I64P, C.POINTER(C.c_int)]),
    "tw_slice_dir_close": (C.c_int, [_P]),
    "tw_box_reader_slices": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _P]),
    "tw_slice_writer_create": (C.c_int, [C.c_char_p, _I64P, C.c_int, C.c_int, C.POINTER(_P)]),
    "tw_slice_writer_close": (C.c_int, [_P]),
    "tw_box_writer_slices": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _P]),
    "tw_marker_file_read": (C.c_int, [C.c_char_p, _MP, C.c_int, C.POINTER(C.c_int)]),
    "tw_marker_file_write": (C.c_int, [C.c_char_p, _MP, C.c_int]),
    "tw_bigimagewarp_files": (C.c_int, [_P, C.POINTER(tw_params), C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p]),
    "tw_server_create": (C.c_int, [_P, C.c_size_t, C.c_int, C.POINTER(_P)]),
    "tw_server_submit": (C.c_int, [_P, C.POINTER(tw_job), C.POINTER(C.c_uint64)]),
    "tw_server_poll": (C.c_int, [_P, C.c_uint64, _DP]),
    "tw_server_wait": (C.c_int, [_P, C.c_uint64, C.c_double, _DP]),
    "tw_server_job_times": (C.c_int, [_P, C.c_uint64, _DP]),
    "tw_server_destroy": (C.c_int, [_P]),
}

_lib = None


def load() -> C.CDLL:
    """Loads the library (building it first if the sources are newer and a
    compiler is present).  Raises if it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    path = LIB_PATH
    override = os.environ.get("TW_LIBRARY")  # an alternative build of the same ABI
    if override:
        path = Path(override)
    elif os.environ.get("TW_NO_BUILD") != "1":
        try:
            from . import build as _build
            _build.build()
        except FileNotFoundError:
            pass
    if not path.exists():
        raise RuntimeError(f"libterawarp_b200.so not found at {path}; run terawarp_b200.build.build()")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib
