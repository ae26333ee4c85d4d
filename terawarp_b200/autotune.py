"""Autotuner for the out-of-core tiled warps.

The tiled engine (tw_imgwarp_smallmemory_tiled / tw_warp_affine_tiled) takes
an output tile shape and a staging depth (device/pinned slots in flight).  The
best pair depends on the volume, the voxel type, the grid spacing and the
host-device link, so it is chosen by timing a few candidates on a sample of
the job -- the corner block of the output, warped with the job's own
landmarks -- and remembered per (kind, volume shape, dtype, grid spacing,
landmark-count bucket, device name).

`tune(run, candidates)` is the search itself: `run(tile_xyz, depth)` returns
seconds, the fastest candidate wins.
"""
from __future__ import annotations

import json
import math
import os
import time
from pathlib import Path
from typing import Callable, Iterable, Sequence

import numpy as np

# (tile x, y, z), staging depth.  TPS tiles are rounded to the grid spacing by
# the engine.  Flat tiles move fewer halo voxels per output voxel in z-major
# volumes; deeper staging hides more of the link.
CANDIDATES: list[tuple[tuple[int, int, int], int]] = [
    ((512, 512, 512), 2),
    ((512, 512, 512), 3),
    ((1024, 1024, 256), 2),
    ((1024, 1024, 256), 3),
    ((2048, 1024, 128), 3),
    ((256, 256, 256), 4),
]


def tune(run: Callable[[tuple, int], float], candidates: Iterable = CANDIDATES, repeats: int = 1):
    """Times every candidate (best of `repeats`) and returns
    (tile_xyz, depth, table) with table = [(tile_xyz, depth, seconds), ...]."""
    table = []
    for tile, depth in candidates:
        best = math.inf
        for _ in range(max(1, repeats)):
            best = min(best, float(run(tuple(tile), int(depth))))
        table.append((tuple(int(v) for v in tile), int(depth), best))
    if not table:
        raise ValueError("no candidates to tune over")
    tile, depth, _ = min(table, key=lambda r: r[2])
    return tile, depth, table


def cache_key(kind: str, shape_zyx: Sequence[int], dtype: str, g: int = 0, n_landmarks: int = 0,
              device: str = "") -> str:
    """Landmark counts fall into power-of-two buckets (the solve and the node
    evaluation scale with them, the tile choice only coarsely)."""
    bucket = 0 if n_landmarks <= 0 else 1 << int(math.ceil(math.log2(n_landmarks)))
    z, y, x = (int(v) for v in shape_zyx)
    return f"{kind}:{x}x{y}x{z}:{dtype}:g{int(g)}:n{bucket}:{device}"


def load_cache(path) -> dict:
    try:
        return json.loads(Path(path).read_text())
    except (OSError, ValueError):
        return {}


def store_cache(path, key: str, tile, depth: int, table) -> None:
    p = Path(path)
    data = load_cache(p)
    data[key] = {"tile": list(tile), "depth": int(depth),
                 "table": [[list(t), int(d), float(s)] for t, d, s in table]}
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(p.suffix + ".tmp")
    tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
    os.replace(tmp, p)


def _sample(src, sample_zyx):
    """Contiguous copy of the source's corner block (pinned when torch)."""
    z, y, x = (min(int(a), int(b)) for a, b in zip(sample_zyx, src.shape))
    crop = src[:z, :y, :x]
    try:
        import torch
        if isinstance(crop, torch.Tensor):
            out = torch.empty(tuple(crop.shape), dtype=crop.dtype, pin_memory=True)
            out.copy_(crop)
            return out
    except ImportError:
        pass
    return np.ascontiguousarray(crop)


def _empty_like(x):
    try:
        import torch
        if isinstance(x, torch.Tensor):
            return torch.empty(tuple(x.shape), dtype=x.dtype, pin_memory=True)
    except ImportError:
        pass
    return np.empty_like(x)


def tune_tiled_tps(ctx, ql_marker_tar, ql_marker_sub, marker_scale: float, g: int, src,
                   sample_zyx=(512, 1024, 1024), candidates=CANDIDATES, cache_path=None, device_name: str = ""):
    """(tile_xyz, depth, table) for imgwarp_smallmemory_tiled on `src` (a host
    volume z, y, x), timed on its corner block; cached when cache_path is set."""
    from . import api

    candidates = list(candidates)
    dtype = "u8" if np.dtype(str(src.dtype).replace("torch.", "")).itemsize == 1 else "u16"
    n = len(np.asarray(ql_marker_tar).reshape(-1, 3))
    key = cache_key("tps", src.shape, dtype, g, n, device_name)
    if cache_path:
        hit = load_cache(cache_path).get(key)
        if hit:
            return tuple(hit["tile"]), int(hit["depth"]), [(tuple(t), d, s) for t, d, s in hit["table"]]
    crop = _sample(src, sample_zyx)
    out = _empty_like(crop)

    def run(tile, depth):
        t0 = time.perf_counter()
        api.imgwarp_smallmemory_tiled(ctx, ql_marker_tar, ql_marker_sub, marker_scale, g, crop, out=out, tile=tile,
                                      depth=depth)
        return time.perf_counter() - t0

    run(candidates[0][0], candidates[0][1])  # the first call pays one-time set-up
    tile, depth, table = tune(run, candidates)
    if cache_path:
        store_cache(cache_path, key, tile, depth, table)
    return tile, depth, table
