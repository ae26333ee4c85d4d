"""The procedural tile source and the checksum sink (CPU only): any two boxes
of the synthetic volume agree where they overlap -- the property a tiled warp
relies on -- and the checksum sink's sums match numpy's."""
import numpy as np
import pytest

from terawarp_b200 import api


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16])
def test_overlapping_boxes_agree(dtype):
    v = api.SyntheticVolume((300, 400, 500), dtype, seed=7, threads=4)
    big = v.read_box((37, 51, 60), (200, 150, 90))
    a = v.read_box((100, 80, 70), (64, 64, 40))
    np.testing.assert_array_equal(a, big[10:50, 29:93, 63:127])
    b = v.read_box((0, 0, 0), (96, 32, 8))
    c = v.read_box((0, 0, 0), (96, 32, 8))
    np.testing.assert_array_equal(b, c)
    # values span the type's range: noise, blobs and fibres are present
    vmax = 255 if dtype == np.uint8 else 4095
    assert big.min() <= 10 and big.max() > vmax // 2 and big.max() <= vmax


def test_boxes_outside_the_volume_are_rejected():
    v = api.SyntheticVolume((10, 20, 30), np.uint16)
    with pytest.raises(api.TeraWarpError):
        v.read_box((25, 0, 0), (10, 5, 5))


def test_checksum_sink_sums():
    rng = np.random.default_rng(3)
    blk = rng.integers(0, 4096, size=(5, 7, 9)).astype(np.uint16)
    c = api.Checksum(np.uint16, threads=2)
    c.write_box((10, 20, 30), blk)
    s, w, n = c.value
    assert s == int(blk.astype(np.uint64).sum()) and n == blk.size
    z, y, x = np.meshgrid(np.arange(30, 35), np.arange(20, 27), np.arange(10, 19), indexing="ij")
    key = ((x.astype(np.uint64) * np.uint64(73856093)) ^ (y.astype(np.uint64) * np.uint64(19349663)) ^
           (z.astype(np.uint64) * np.uint64(83492791)))
    assert w == int((blk.astype(np.uint64) * key).sum(dtype=np.uint64))
