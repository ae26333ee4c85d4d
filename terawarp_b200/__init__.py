"""terawarp_b200 -- B200-native (sm_100a) implementation of TeraWarp's warp
path: FP64 TPS landmark solve, FP32 compensated TPS evaluation at the
control-grid nodes, fused cubic B-spline expansion + trilinear resampling of
uint8/uint16 volumes, affine / rotation / translation / scaling warps, and
pinned double-buffered host<->HBM streaming, behind a C ABI
(include/terawarp_b200.h, libterawarp_b200.so).  `terawarp_b200.api` mirrors
the reference's operator functions over that ABI.
"""
from .api import (Context, TeraWarpError, TPS, bigimagewarp, downsample_factor, downsample_image, fit_affine,
                  fit_affine_noalloc, grid_size, imgwarp_smallmemory_image, make_affine, output_size, params, q_imagewarp_affine_image,
                  tps_eval_grid, tps_solve, warp_affine_device, warp_tps_device)

__all__ = [
    "Context", "TeraWarpError", "TPS", "bigimagewarp", "downsample_factor", "downsample_image", "fit_affine",
    "fit_affine_noalloc", "grid_size", "imgwarp_smallmemory_image", "make_affine", "output_size", "params", "q_imagewarp_affine_image",
    "tps_eval_grid", "tps_solve", "warp_affine_device", "warp_tps_device",
]
