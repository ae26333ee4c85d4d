"""Host-side argument checks of the Python mirror, made before any library
call (CPU only: the context is a stand-in whose library must never be
reached)."""
import numpy as np
import pytest

from terawarp_b200 import api


class _NoLib:
    def __getattr__(self, name):
        raise AssertionError(f"{name} was called although the arguments are invalid")


class _FakeCtx:
    handle = None
    device = 0
    lib = _NoLib()


@pytest.mark.parametrize("fn", [api.fit_affine, api.fit_affine_noalloc])
def test_affine_fit_rejects_unequal_landmark_sets(fn):
    tar = np.zeros((8, 3), np.float32)
    sub = np.zeros((5, 3), np.float32)
    with pytest.raises(ValueError, match="differ in length"):
        fn(_FakeCtx(), tar, sub)
    # the check applies after the (-1, 3) reshape: 24 flat values are 8 points
    with pytest.raises(ValueError, match="8 vs 5"):
        fn(_FakeCtx(), tar.reshape(-1), sub)


def test_tps_solve_rejects_unequal_landmark_sets():
    with pytest.raises(ValueError, match="differ in length"):
        api.tps_solve(_FakeCtx(), np.zeros((10, 3)), np.zeros((9, 3)))


def test_tiled_rejects_unequal_landmark_sets():
    vol = np.zeros((4, 4, 4), np.uint8)
    with pytest.raises(ValueError, match="differ in length"):
        api.imgwarp_smallmemory_tiled(_FakeCtx(), np.zeros((6, 3)), np.zeros((7, 3)), 1.0, 4, vol, out=vol)
