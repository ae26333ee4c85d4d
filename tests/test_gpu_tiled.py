"""Tiled out-of-core streaming (imgwarp_smallmemory_CYF / q_imagewarp_affine_cyf
analogues): the tiled result must equal the whole-volume result, for every
kind of tile source/sink (built-in host reader on pageable memory, strided
DMA on pinned memory, Python callbacks) and for uneven edge tiles."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import terawarp_b200 as tw
from oracle import oracle as O
from terawarp_b200 import api, synth

pytestmark = pytest.mark.gpu


def agree(a, b, frac=0.9999):
    d = np.abs(np.asarray(a, np.int64) - np.asarray(b, np.int64))
    assert (d <= 1).mean() >= frac, (d <= 1).mean()
    return d


@pytest.fixture(scope="module")
def case():
    c = synth.large_tps_case(seed=21, device="cpu", shape_zyx=(96, 300, 520), n=80, g=8, n_blobs=300, n_fibres=40)
    return c.vol.numpy(), c.marker_sub, c.marker_tar


def test_tiled_tps_equals_whole_volume(ctx, case):
    img, sub, tar = case
    whole = tw.imgwarp_smallmemory_image(ctx, sub, tar, 8, 8, 8, 1, 0, img)
    # same node grid, the same unit frames and the same per-voxel arithmetic
    tiled = api.imgwarp_smallmemory_tiled(ctx, sub, tar, 1.0, 8, img, tile=(256, 256, 64), depth=2)
    np.testing.assert_array_equal(tiled, whole)


def test_tiled_tps_uneven_tiles_and_pinned_dma(ctx, case):
    img, sub, tar = case
    whole = tw.imgwarp_smallmemory_image(ctx, sub, tar, 8, 8, 8, 1, 0, img)
    src = torch.from_numpy(img).pin_memory()
    out = torch.empty_like(src).pin_memory()
    api.imgwarp_smallmemory_tiled(ctx, sub, tar, 1.0, 8, src, out=out, tile=(96, 72, 40), depth=3)
    agree(out.numpy(), whole)
    ref = O.imgwarp_smallmemory_image(sub, tar, 8, img)
    agree(out.numpy(), ref)


def test_tiled_tps_python_callbacks(ctx):
    c = synth.plain_tps_case(device="cpu", shape_zyx=(40, 64, 96), n=16, g=8)
    img = c.vol.numpy()
    out = np.zeros_like(img)

    def rd(x0, y0, z0, nx, ny, nz):
        return img[z0:z0 + nz, y0:y0 + ny, x0:x0 + nx]

    def wr(x0, y0, z0, blk):
        out[z0:z0 + blk.shape[0], y0:y0 + blk.shape[1], x0:x0 + blk.shape[2]] = blk

    api.imgwarp_smallmemory_tiled(ctx, c.marker_sub, c.marker_tar, 1.0, 8, img, tile=(64, 32, 16), read_fn=rd,
                                  write_fn=wr)
    whole = tw.imgwarp_smallmemory_image(ctx, c.marker_sub, c.marker_tar, 8, 8, 8, 1, 0, img)
    agree(out, whole)


def test_tiled_marker_scale(ctx):
    # the reference's tiled path scales both marker sets by 4
    # (q_imgwarp_tps_quicksmallmemory.cpp:1194-1203)
    c = synth.plain_tps_case(device="cpu", shape_zyx=(48, 96, 128), n=20, g=8)
    img = c.vol.numpy()
    out = api.imgwarp_smallmemory_tiled(ctx, c.marker_sub / 4, c.marker_tar / 4, 4.0, 8, img, tile=(256, 256, 48))
    whole = tw.imgwarp_smallmemory_image(ctx, c.marker_sub, c.marker_tar, 8, 8, 8, 1, 0, img)
    agree(out, whole)


def test_tiled_callback_failure_is_reported(ctx):
    c = synth.plain_tps_case(device="cpu", shape_zyx=(32, 48, 64), n=12, g=8)
    img = c.vol.numpy()

    def rd(*a):
        raise IOError("disk gone")

    with pytest.raises(tw.TeraWarpError) as e:
        api.imgwarp_smallmemory_tiled(ctx, c.marker_sub, c.marker_tar, 1.0, 8, img, tile=(64, 48, 32), read_fn=rd,
                                      write_fn=lambda *a: None)
    assert e.value.status == 6  # TW_ERR_IO


@pytest.mark.parametrize("out_shape", [(60, 90, 130), (71, 45, 200)])
def test_tiled_affine_matches_device_path(ctx, out_shape):
    rng = np.random.default_rng(5)
    img = rng.integers(0, 4096, size=(60, 90, 130)).astype(np.uint16)
    M = synth.random_affine(9, (130, 90, 60), trans=6.0)
    out = api.warp_affine_tiled(ctx, M, img, out_shape, tile=(64, 48, 24), depth=2)
    src = torch.from_numpy(img).cuda()
    dst = torch.empty(out_shape, dtype=torch.uint16, device="cuda")
    tw.warp_affine_device(ctx, M, src, dst)
    torch.cuda.synchronize()
    agree(out, dst.cpu().numpy())
    agree(out, O.affine_warp(img, M, out_shape))


def test_autotuned_tile_choice_gives_the_whole_volume_result(ctx):
    """The autotuner times real tiled runs on the corner block; whatever it
    picks, the tiled warp equals the whole-volume warp."""
    from terawarp_b200 import autotune
    shape = (40, 96, 136)
    rng = np.random.default_rng(21)
    vol = rng.integers(0, 4096, size=shape).astype(np.uint16)
    sub, tar = synth.lattice_landmarks(shape[::-1], 40, 22, margin=6.0)
    cands = [((64, 64, 32), 2), ((32, 32, 16), 3), ((128, 96, 40), 2)]
    tile, depth, table = autotune.tune_tiled_tps(ctx, sub, tar, 1.0, 8, vol, sample_zyx=(32, 64, 96),
                                                 candidates=cands)
    assert (tile, depth) in [(t, d) for t, d in cands] and len(table) == 3
    tiled = api.imgwarp_smallmemory_tiled(ctx, sub, tar, 1.0, 8, vol, tile=tile, depth=depth)
    whole = tw.imgwarp_smallmemory_image(ctx, sub, tar, 8, 8, 8, 1, 0, vol)
    np.testing.assert_array_equal(tiled, whole)


def test_edge_tiles_are_batched_and_equal_the_whole_volume(ctx, case):
    """Uneven edge tiles are warped in shared launches (fewer resample launches
    than tiles) and the tiled result equals the whole-volume result voxel for
    voxel: tiles start on the whole volume's resample-unit boundaries."""
    img, sub, tar = case                     # 520 x 300 x 96 u16, g = 8
    whole = tw.imgwarp_smallmemory_image(ctx, sub, tar, 8, 8, 8, 1, 0, img)
    # launches of one solve + node grid, to subtract from the tiled call's count
    n0 = ctx.kernel_launches
    t = tw.tps_solve(ctx, tar, sub)
    solve_launches = ctx.kernel_launches - n0
    t.close()
    # kernel launches of one resample pass (planning + staged + gather kernels
    # for a stageable trilinear job) on a small device volume of the same kind
    t = tw.tps_solve(ctx, tar, sub)
    small = torch.from_numpy(np.ascontiguousarray(img[:16, :64, :128])).cuda()
    nodes = tw.tps_eval_grid(ctx, t, (tw.grid_size(128, 8), tw.grid_size(64, 8), tw.grid_size(16, 8)), 8)
    out = torch.empty_like(small)
    n1 = ctx.kernel_launches
    tw.warp_tps_device(ctx, nodes, 8, small, out)
    per_pass = ctx.kernel_launches - n1
    t.close()
    before = ctx.kernel_launches
    tiled = api.imgwarp_smallmemory_tiled(ctx, sub, tar, 1.0, 8, img, tile=(256, 128, 64), depth=2)
    resample_launches = ctx.kernel_launches - before - solve_launches - 2  # node grid + tile hulls
    assert resample_launches % per_pass == 0
    passes = resample_launches // per_pass
    # tiles: x 256, 256, 8; y 128, 128, 44; z 64, 32 -> 18 tiles, 4 of them full
    ntiles, nfull = 18, 4
    assert passes < ntiles
    assert passes >= nfull + 1
    np.testing.assert_array_equal(tiled, whole)
