"""The seeded synthetic inputs: a z-range of a volume is those planes of the
whole volume, so the CPU baseline can time exactly the input the GPU warps.
CPU only."""
import torch

from terawarp_b200 import synth


def test_z_range_reproduces_planes_of_the_whole_volume():
    full = synth.blob_volume((40, 64, 80), "u16", 5, n_blobs=60, n_fibres=20)
    for z0, z1 in [(0, 8), (7, 19), (39, 40)]:
        part = synth.blob_volume((40, 64, 80), "u16", 5, n_blobs=60, n_fibres=20, z_range=(z0, z1))
        assert torch.equal(full[z0:z1], part)


def test_large_case_landmarks_do_not_depend_on_z_range():
    a = synth.large_tps_case(9, "cpu", shape_zyx=(64, 96, 128), n=50, n_blobs=40, n_fibres=5)
    b = synth.large_tps_case(9, "cpu", shape_zyx=(64, 96, 128), n=50, n_blobs=40, n_fibres=5, z_range=(10, 14))
    assert (a.marker_sub == b.marker_sub).all() and (a.marker_tar == b.marker_tar).all()
    assert torch.equal(a.vol[10:14], b.vol)
