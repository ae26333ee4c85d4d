"""The plugin's command on files (tw_bigimagewarp_files, plugin_Bigimagewarp.cpp:
123-336): a .v3draw volume or a directory of per-Z slices in, the warped
volume out -- for slices, tiles written straight into the output slice files
(no stitching pass) -- plus the downsampled preview.  Each output must equal
the in-memory warp of the same volume, voxel for voxel."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import terawarp_b200 as tw
from terawarp_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    c = synth.large_tps_case(seed=31, device="cpu", shape_zyx=(80, 150, 260), n=60, g=8, n_blobs=200, n_fibres=20)
    return c.vol.numpy(), c.marker_sub, c.marker_tar


def write_inputs(tmp_path, vol, sub, tar, slices: bool, marker_div: float = 1.0):
    api.write_markers(tmp_path / "sub.marker", sub / marker_div)
    api.write_markers(tmp_path / "tar.marker", tar / marker_div)
    if slices:
        d = tmp_path / "brain"
        os.makedirs(d)
        for z in range(vol.shape[0]):
            api.v3draw_write(d / f"{z:05d}.v3draw", vol[z:z + 1])
        return str(d)
    p = tmp_path / "brain.v3draw"
    api.v3draw_write(p, vol)
    return str(p)


def test_v3draw_tps_and_downsample(ctx, case, tmp_path):
    vol, sub, tar = case
    img = write_inputs(tmp_path, vol, sub, tar, slices=False)
    out = tmp_path / "out"
    os.makedirs(out)
    api.bigimagewarp_files(ctx, img, str(tmp_path / "sub.marker"), str(tmp_path / "tar.marker"), str(out),
                           downsample_mode=1, warp_mode=0, deformation_mode=1, grid_spacing=8)
    got = api.v3draw_read(out / "brain_stps.v3draw")
    # the markers went through the text file: compare with the same values
    sub_f, tar_f = api.read_markers(tmp_path / "sub.marker"), api.read_markers(tmp_path / "tar.marker")
    want = tw.bigimagewarp(ctx, vol, sub_f, tar_f, warp_mode=0, deformation_mode=1, grid_spacing=8)
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(api.v3draw_read(out / "brain_stps_downsample.v3draw"), tw.downsample_image(ctx, want))


def test_v3draw_affine(ctx, case, tmp_path):
    vol, sub, tar = case
    img = write_inputs(tmp_path, vol, sub, tar, slices=False)
    out = tmp_path / "out"
    os.makedirs(out)
    api.bigimagewarp_files(ctx, img, str(tmp_path / "sub.marker"), str(tmp_path / "tar.marker"), str(out),
                           warp_mode=0, deformation_mode=0)
    sub_f, tar_f = api.read_markers(tmp_path / "sub.marker"), api.read_markers(tmp_path / "tar.marker")
    want = tw.bigimagewarp(ctx, vol, sub_f, tar_f, warp_mode=0, deformation_mode=0)
    np.testing.assert_array_equal(api.v3draw_read(out / "brain_affine.v3draw"), want)


def test_slice_directory_tps_writes_slices_equal_to_the_whole_volume_warp(ctx, case, tmp_path):
    """The reference's tiled path reads markers placed on a 4x downsampled
    image and scales them by 4 (q_imgwarp_tps_quicksmallmemory.cpp:1194-1203);
    the output slices must equal the whole-volume warp with the scaled
    markers."""
    vol, sub, tar = case
    img = write_inputs(tmp_path, vol, sub, tar, slices=True, marker_div=4.0)
    out = tmp_path / "out"
    os.makedirs(out)
    api.bigimagewarp_files(ctx, img, str(tmp_path / "sub.marker"), str(tmp_path / "tar.marker"), str(out),
                           downsample_mode=1, warp_mode=0, deformation_mode=1, grid_spacing=8)
    sub_f = api.read_markers(tmp_path / "sub.marker").astype(np.float64) * 4
    tar_f = api.read_markers(tmp_path / "tar.marker").astype(np.float64) * 4
    want = tw.imgwarp_smallmemory_image(ctx, sub_f, tar_f, 8, 8, 8, 1, 0, vol)
    got = api.read_slices(out / "brain_stps_slice")
    assert sorted(os.listdir(out / "brain_stps_slice"))[:2] == ["0000000.raw", "0000010.raw"]
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(api.read_slices(out / "brain_stps_downsample_slice"), tw.downsample_image(ctx, want))


def test_slice_directory_rotation(ctx, case, tmp_path):
    vol, sub, tar = case
    img = write_inputs(tmp_path, vol, sub, tar, slices=True)
    out = tmp_path / "out"
    os.makedirs(out)
    api.bigimagewarp_files(ctx, img, None, None, str(out), warp_mode=1, deformation_mode=0, para=(5.0, -8.0, 12.0))
    want = tw.bigimagewarp(ctx, vol, warp_mode=1, deformation_mode=0, para=(5.0, -8.0, 12.0))
    got = api.read_slices(out / "brain_rotation_slice")
    d = np.abs(got.astype(np.int64) - want.astype(np.int64))
    # the tiled affine path starts its FP32 increments at each tile's bricks
    assert (d <= 1).mean() >= 0.9999
