"""Parity with the FP64 oracle at the benchmark configurations' full sizes,
through the C ABI.

  large TPS    2048 x 2048 x 1024 uint16, 2000 landmarks on a jittered
               lattice (sinusoidal displacement <= 12 voxels + N(0, 1)):
               node displacement over the whole control grid at spacing 8
               and 16 (max <= 0.01 voxel, RMS <= 0.002 voxel), and output
               intensities within +-1 level on >= 99.99 % of the voxels of
               seeded 512^3 tiles of the whole-volume warp (the two corner
               tiles and two interior ones), the oracle running its own FP64
               solve and node grid
  affine       1024 x 1024 x 512 uint16, matrix fitted from 32 landmark pairs:
               the matrix against the oracle's fit, the whole output volume
               within +-1 level on >= 99.99 % of voxels
  solve        4096 landmark pairs (the terabyte and serving configurations'
               largest count) against the oracle's FP64 solve

The oracle restates the reference's CPU path (q_imgwarp_tps_quicksmallmemory.cpp
:377-661 solve and grid, :85-203 B-spline and warp; q_warp_affine_tps.cpp
:649-731 fit, :1373-1437 warp).  Host memory: ~17 GB; device: ~17 GB.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import terawarp_b200 as tw
from oracle import oracle as O
from terawarp_b200 import synth

pytestmark = pytest.mark.gpu

INT_TOL_FRAC = 0.9999
NODE_MAX = 0.01
NODE_RMS = 0.002
SHAPE = (1024, 2048, 2048)      # z, y, x
TILE = 512


def _within(a, b):
    d = np.abs(np.asarray(a, np.int64) - np.asarray(b, np.int64))
    return float((d <= 1).mean()), float((d == 0).mean()), int(d.max())


@pytest.fixture(scope="module")
def large():
    case = synth.large_tps_case(1237, "cuda", shape_zyx=SHAPE, n=2000, g=16)
    src_h = case.vol.cpu().numpy()
    # the reference's argument order: centres = target markers, values = subject markers
    c, d = O.tps_solve(case.marker_tar, case.marker_sub)
    yield {"case": case, "src_h": src_h, "c": c, "d": d, "grids": {}}
    del case


def _gpu_nodes(ctx, case, g):
    Z, Y, X = SHAPE
    gsz = (tw.grid_size(X, g), tw.grid_size(Y, g), tw.grid_size(Z, g))
    t = tw.tps_solve(ctx, case.marker_tar, case.marker_sub)
    nodes = tw.tps_eval_grid(ctx, t, gsz, g)
    torch.cuda.synchronize()
    t.close()
    return gsz, nodes


def _oracle_grid(large, g):
    if g not in large["grids"]:
        Z, Y, X = SHAPE
        gsz = (O.grid_size(X, g), O.grid_size(Y, g), O.grid_size(Z, g))
        large["grids"][g] = O.tps_grid(large["case"].marker_tar, large["c"], large["d"], gsz, g)
    return large["grids"][g]


@pytest.mark.parametrize("g", [16, 8])
def test_large_tps_node_displacement_over_the_whole_grid(ctx, large, g):
    gsz, nodes = _gpu_nodes(ctx, large["case"], g)
    got = nodes.cpu().numpy()[..., :3].astype(np.float64)
    ref = _oracle_grid(large, g).astype(np.float64)
    assert got.shape == ref.shape
    err = np.abs(got - ref)
    emax, erms = float(err.max()), float(np.sqrt((err ** 2).mean()))
    print(f"g={g}: {ref.shape[0] * ref.shape[1] * ref.shape[2]} nodes, max {emax:.2e}, rms {erms:.2e} voxel")
    assert emax <= NODE_MAX, emax
    assert erms <= NODE_RMS, erms


def _tiles(seed=2024):
    Z, Y, X = SHAPE
    rng = np.random.default_rng(seed)
    corners = [(0, 0, 0), (X - TILE, Y - TILE, Z - TILE)]
    inner = [tuple(int(v) for v in rng.integers(1, [(X - TILE) // 16, (Y - TILE) // 16, (Z - TILE) // 16]) * 16)
             for _ in range(2)]
    return corners + inner


@pytest.mark.parametrize("g", [16, 8])
def test_large_tps_intensities_on_tiles_of_the_whole_volume(ctx, large, g):
    case = large["case"]
    gsz, nodes = _gpu_nodes(ctx, case, g)
    dst = torch.empty_like(case.vol)
    tw.warp_tps_device(ctx, nodes, g, case.vol, dst)
    torch.cuda.synchronize()
    del nodes
    df = _oracle_grid(large, g)
    for (x0, y0, z0) in _tiles():
        ref = O.tps_warp_box(large["src_h"], df, g, (x0, y0, z0), (TILE, TILE, TILE))
        got = dst[z0:z0 + TILE, y0:y0 + TILE, x0:x0 + TILE].cpu().numpy()
        within, exact, dmax = _within(got, ref)
        print(f"g={g} tile {(x0, y0, z0)}: within+-1 {within:.7f}, exact {exact:.5f}, max diff {dmax}")
        assert within >= INT_TOL_FRAC, (x0, y0, z0, within, dmax)
    del dst


def test_affine_configuration_whole_volume(ctx):
    case = synth.affine_case(device="cuda")
    M = tw.fit_affine(ctx, case.marker_tar, case.marker_sub)
    M0 = O.affine_fit(case.marker_tar, case.marker_sub)
    np.testing.assert_allclose(M, M0, atol=1e-9, rtol=0)
    dst = torch.empty_like(case.vol)
    tw.warp_affine_device(ctx, M, case.vol, dst)
    torch.cuda.synchronize()
    src_h = case.vol.cpu().numpy()
    ref = O.affine_warp(src_h, M0)
    within, exact, dmax = _within(dst.cpu().numpy(), ref)
    print(f"affine 1024x1024x512: within+-1 {within:.7f}, exact {exact:.5f}, max diff {dmax}")
    assert within >= INT_TOL_FRAC
    assert (ref == 0).mean() > 0.001  # the rotation moves part of the output outside the subject


def test_solve_at_4096_landmarks(ctx):
    sub, tar = synth.lattice_landmarks((16384, 16384, 4096), 4096, 1244)
    t = tw.tps_solve(ctx, tar, sub)
    c, d = t.coeffs()
    t.close()
    c0, d0 = O.tps_solve(tar, sub)
    np.testing.assert_allclose(c, c0, atol=1e-7 * max(1.0, np.abs(c0).max()), rtol=0)
    np.testing.assert_allclose(d, d0, atol=1e-7 * max(1.0, np.abs(d0).max()), rtol=0)
