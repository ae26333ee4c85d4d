"""The FP64 oracle against the golden fixtures (an independent numpy
restatement, tests/golden/make_golden.py) and against known answers the
mathematics dictates.  CPU only."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

G = np.load(Path(__file__).resolve().parent / "golden" / "golden_small.npz")


def test_solve_matches_bordered_golden():
    c, d = O.tps_solve(G["tps_ctr"], G["tps_val"])
    np.testing.assert_allclose(c, G["tps_c"], atol=1e-10)
    np.testing.assert_allclose(d, G["tps_d"], atol=1e-9)


@pytest.mark.parametrize("g", [4, 8])
def test_grid_matches_golden(g):
    src = G["tps_src"]
    Z, Y, X = src.shape
    c, d = O.tps_solve(G["tps_ctr"], G["tps_val"])
    gsz = (O.grid_size(X, g), O.grid_size(Y, g), O.grid_size(Z, g))
    df = O.tps_grid(G["tps_ctr"], c, d, gsz, g)
    np.testing.assert_allclose(df, G[f"tps_df_g{g}"], atol=2e-5)


@pytest.mark.parametrize("g", [4, 8])
def test_warp_matches_golden(g):
    src = G["tps_src"]
    out = O.tps_warp(src, G[f"tps_df_g{g}"], g, 0, threads=1)
    ref = G[f"tps_out_g{g}"]
    diff = np.abs(out.astype(int) - ref.astype(int))
    assert diff.max() <= 1
    assert (diff == 0).mean() >= 0.999


def test_full_pipeline_matches_golden():
    src = G["tps_src"]
    out = O.imgwarp_smallmemory_image(G["tps_val"], G["tps_ctr"], 4, src)
    diff = np.abs(out.astype(int) - G["tps_out_g4"].astype(int))
    assert diff.max() <= 1 and (diff == 0).mean() >= 0.999


def test_affine_fit_and_warp_match_golden():
    M = O.affine_fit(G["aff_tar"], G["aff_sub"])
    np.testing.assert_allclose(M, G["aff_M"], atol=1e-8)
    out = O.affine_warp(G["aff_src"], G["aff_M"], (20, 24, 28))
    diff = np.abs(out.astype(int) - G["aff_out"].astype(int))
    assert diff.max() <= 1 and (diff == 0).mean() >= 0.999


def _vol(shape, dtype, seed=0):
    rng = np.random.default_rng(seed)
    hi = 256 if dtype == np.uint8 else 4096
    return rng.integers(0, hi, size=shape).astype(dtype)


def test_identity_landmarks_copy_volume():
    # TPS with target == subject is the identity: every voxel samples itself
    src = _vol((20, 24, 28), np.uint8)
    rng = np.random.default_rng(1)
    pts = rng.uniform(2, 18, size=(10, 3)).astype(np.float32)
    out = O.imgwarp_smallmemory_image(pts, pts, 4, src)
    # interior voxels are copied exactly; on the outer face the solve's
    # 1e-15 residual can put q a hair outside [0, sz-1], which the
    # reference's bounds test turns into 0
    np.testing.assert_array_equal(out[1:-1, 1:-1, 1:-1], src[1:-1, 1:-1, 1:-1])
    assert np.all((out == src) | (out == 0))


def test_affine_landmarks_give_zero_nonaffine_part():
    rng = np.random.default_rng(2)
    ctr = rng.uniform(0, 100, size=(30, 3)).astype(np.float32)
    A = np.array([[1.02, 0.01, -0.02], [0.0, 0.98, 0.03], [0.01, -0.01, 1.01]])
    t = np.array([3.0, -2.0, 1.5])
    val = (ctr.astype(np.float64) @ A.T + t).astype(np.float32)
    c, d = O.tps_solve(ctr, val)
    assert np.abs(c).max() < 1e-5
    np.testing.assert_allclose(d[1:, 1:], A.T, atol=1e-5)
    np.testing.assert_allclose(d[0, 1:], t, atol=1e-3)


def test_integer_shift_affine_is_exact_copy():
    src = _vol((16, 18, 20), np.uint16)
    M = np.eye(4)
    M[:3, 3] = [2, -1, 3]
    out = O.affine_warp(src, M)
    ref = np.zeros_like(src)
    # out(x,y,z) = src(x+2, y-1, z+3) where in range
    ref[0:13, 1:18, 0:18] = src[3:16, 0:17, 2:20]
    np.testing.assert_array_equal(out, ref)


def test_out_of_bounds_samples_are_zero():
    src = np.full((10, 12, 14), 200, np.uint8)
    M = np.eye(4)
    M[0, 3] = 100.0  # every sample lands right of the volume
    assert O.affine_warp(src, M).max() == 0


def test_bspline_reproduces_constant_and_linear_fields():
    # a node field that is constant (or linear in the node position) is
    # reproduced exactly by the cubic B-spline: partition of unity and
    # linear precision of the uniform cubic B-spline
    for g in (4, 8, 16):
        tb = np.zeros((g, 4))
        O.load().or_bspline_tb(g, tb)
        np.testing.assert_allclose(tb.sum(1), 1.0, atol=1e-14)
        t = np.arange(g) / g
        np.testing.assert_allclose(tb @ np.array([-1.0, 0.0, 1.0, 2.0]), t, atol=1e-14)


def test_nearest_neighbour_rule():
    src = _vol((8, 9, 10), np.uint8, 3)
    M = np.eye(4)
    M[:3, 3] = [0.4, 0.6, -0.2]
    out = O.affine_warp(src, M, interp=1)
    # (long)(q + 0.5) with q = p + shift, clamped to sz - 1; OOB (q < 0) -> 0
    z, y, x = np.meshgrid(np.arange(8), np.arange(9), np.arange(10), indexing="ij")
    qx, qy, qz = x + 0.4, y + 0.6, z - 0.2
    ok = (qx <= 9) & (qy <= 8) & (qz >= 0) & (qz <= 7)
    nx = np.minimum((qx + 0.5).astype(int), 9)
    ny = np.minimum((qy + 0.5).astype(int), 8)
    nz = np.minimum((qz + 0.5).astype(int), 7)
    ref = np.where(ok, src[nz, ny, nx], 0)
    np.testing.assert_array_equal(out, ref)


def test_downsample_factor_rule():
    assert O.downsample_factor((600, 100, 100)) == 1
    assert O.downsample_factor((899, 100, 100)) == 1
    assert O.downsample_factor((900, 100, 100)) == 2
    assert O.downsample_factor((100, 100, 18052)) == 30


def test_degenerate_landmarks_rejected():
    ctr = np.zeros((6, 3), np.float32)
    ctr[:, 0] = np.arange(6)
    ctr[:, 1] = np.arange(6) * 2.0  # collinear
    with pytest.raises(RuntimeError):
        O.tps_solve(ctr, ctr)


def test_parallel_and_serial_oracle_agree():
    src = _vol((24, 20, 30), np.uint8, 5)
    rng = np.random.default_rng(6)
    s = rng.uniform(2, 18, size=(9, 3)).astype(np.float32)
    t = (s + rng.normal(0, 1.0, size=s.shape)).astype(np.float32)
    a = O.imgwarp_smallmemory_image(t, s, 4, src, threads=1)
    b = O.imgwarp_smallmemory_image(t, s, 4, src, threads=0)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("box", [((13, 7, 5), (30, 20, 17)), ((0, 0, 0), (60, 50, 40)), ((59, 49, 39), (1, 1, 1))])
def test_box_warp_equals_the_whole_warp_on_that_box(box):
    rng = np.random.default_rng(0)
    src = rng.integers(0, 4096, size=(40, 50, 60)).astype(np.uint16)
    tar = rng.uniform(3, [57, 47, 37], size=(20, 3)).astype(np.float32)
    sub = (tar + rng.normal(0, 3, size=tar.shape)).astype(np.float32)
    c, d = O.tps_solve(tar, sub)
    g = 8
    df = O.tps_grid(tar, c, d, (O.grid_size(60, g), O.grid_size(50, g), O.grid_size(40, g)), g)
    (ox, oy, oz), (nx, ny, nz) = box
    full = O.tps_warp(src, df, g)
    np.testing.assert_array_equal(O.tps_warp_box(src, df, g, (ox, oy, oz), (nx, ny, nz)),
                                  full[oz:oz + nz, oy:oy + ny, ox:ox + nx])
