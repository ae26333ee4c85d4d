"""Tile-shape / staging-depth choice for the out-of-core tiled TPS warp.

The tuner itself is in the library (tw_tune_tiled_tps): it solves the job's
landmarks and evaluates its node grid once, times each candidate (tile
shape, staging depth) on the job's corner block through the tiled engine,
and remembers the winner per (volume dims, dtype, grid spacing, landmark
count rounded up to a power of two, device name) for the process and, when
a cache file is given, across processes.  This module is its Python caller.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

# The library's default candidates: (tile x, y, z), staging depth.  TPS tiles
# are rounded to whole resample units by the engine.  Flat tiles move fewer
# halo voxels per output voxel; deeper staging hides more of the link.
CANDIDATES: list[tuple[tuple[int, int, int], int]] = [
    ((512, 512, 512), 2),
    ((512, 512, 512), 3),
    ((1024, 1024, 256), 2),
    ((1024, 1024, 256), 3),
    ((2048, 1024, 128), 3),
    ((256, 256, 256), 4),
]


def _cands(candidates):
    arr = (L.tw_tile_candidate * len(candidates))()
    for i, (tile, depth) in enumerate(candidates):
        for a in range(3):
            arr[i].tile[a] = int(tile[a])
        arr[i].staging_depth = int(depth)
    return arr


def tune_tiled_tps(ctx, ql_marker_tar, ql_marker_sub, marker_scale: float, g: int, src,
                   sample_zyx=(512, 1024, 1024), candidates=CANDIDATES, cache_path=None):
    """(tile_xyz, depth, table) for imgwarp_smallmemory_tiled on `src` (a host
    volume z, y, x or a SliceDir); table = [(tile_xyz, depth, seconds)] of the
    candidates timed now (empty when the choice came from a cache)."""
    from . import api

    candidates = list(candidates)
    n = api._pair_count(ql_marker_tar, ql_marker_sub, "tune_tiled_tps")
    rd, ru, _, _, keep = api._box_io(src, None, None, lambda *a: None)
    arr = _cands(candidates)
    best = L.tw_tile_opts()
    smp = (C.c_int64 * 3)(int(sample_zyx[2]), int(sample_zyx[1]), int(sample_zyx[0]))
    st = L.load().tw_tune_tiled_tps(ctx.handle if ctx is not None else None, api._markers(ql_marker_tar),
                                    api._markers(ql_marker_sub), n, float(marker_scale), int(g), api._src_dtype(src),
                                    api._src_sz3(src), rd, ru, arr, len(candidates), smp,
                                    str(cache_path).encode() if cache_path else None, C.byref(best))
    del keep
    api._check(st, ctx, "tw_tune_tiled_tps")
    tile = tuple(int(best.tile[a]) for a in range(3))
    table = [(tuple(int(arr[i].tile[a]) for a in range(3)), int(arr[i].staging_depth), float(arr[i].seconds))
             for i in range(len(candidates)) if arr[i].seconds > 0]
    return tile, int(best.staging_depth), table


def cached_choice(shape_zyx, dtype, g: int, n_landmarks: int, cache_path):
    """The cached (tile_xyz, depth) for a job from the cache file alone (no
    GPU, device name empty), or None."""
    best = L.tw_tile_opts()
    z, y, x = (int(v) for v in shape_zyx)
    sz = (C.c_int64 * 3)(x, y, z)
    code = L.TW_U8 if np.dtype(dtype) == np.uint8 else L.TW_U16
    st = L.load().tw_tune_tiled_tps(None, None, None, int(n_landmarks), 1.0, int(g), code, sz, L.READ_BOX(0), None,
                                    None, 0, None, str(cache_path).encode(), C.byref(best))
    if st == L.TW_ERR_NOT_READY:
        return None
    if st != L.TW_OK:
        raise RuntimeError(f"tw_tune_tiled_tps: status {st}")
    return tuple(int(best.tile[a]) for a in range(3)), int(best.staging_depth)
