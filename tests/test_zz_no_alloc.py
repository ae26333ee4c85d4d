"""tw_fit_affine_noalloc: the affine fit with its scratch in a fixed device
array.  It must return what tw_fit_affine returns, call after call, reject
landmark counts beyond its limit, and leave free device memory unchanged.

The file name sorts last so that these tests also run after every other GPU
test in one session (the scratch array is shared by all calls on a device)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import terawarp_b200 as tw
from terawarp_b200 import api, synth

pytestmark = pytest.mark.gpu

# same kernel and FP64 arithmetic as tw_fit_affine: the matrices agree exactly;
# the tolerance only allows for a different summation order should one appear
ATOL = 1e-12


def landmark_set(seed, n, shape_xyz=(300, 200, 100)):
    M = synth.random_affine(seed, shape_xyz)
    sub, tar = synth.affine_landmarks(M, shape_xyz, n, seed + 1)
    return tar, sub


@pytest.mark.parametrize("n", [4, 32, 1000, api.FIT_AFFINE_NOALLOC_MAX])
def test_two_calls_in_a_row_match_fit_affine(ctx, n):
    sets = [landmark_set(11, n), landmark_set(23, n)]
    got = [tw.fit_affine_noalloc(ctx, tar, sub) for tar, sub in sets]
    want = [tw.fit_affine(ctx, tar, sub) for tar, sub in sets]
    for g, w in zip(got, want):
        np.testing.assert_allclose(g, w, rtol=0, atol=ATOL)
    assert not np.allclose(got[0], got[1])  # the second call did not reuse the first result


def test_rejects_more_landmarks_than_its_limit(ctx):
    tar, sub = landmark_set(5, api.FIT_AFFINE_NOALLOC_MAX + 1)
    with pytest.raises(tw.TeraWarpError) as e:
        tw.fit_affine_noalloc(ctx, tar, sub)
    assert e.value.status == 1  # TW_ERR_ARG
    assert "4096" in str(e.value)
    tar, sub = landmark_set(5, 3)
    with pytest.raises(tw.TeraWarpError) as e:
        tw.fit_affine_noalloc(ctx, tar, sub)
    assert e.value.status == 1
    # the context is still usable
    tar, sub = landmark_set(6, 64)
    np.testing.assert_allclose(tw.fit_affine_noalloc(ctx, tar, sub), tw.fit_affine(ctx, tar, sub), rtol=0, atol=ATOL)


def test_allocates_no_device_memory(ctx):
    tar, sub = landmark_set(7, 500)
    tw.fit_affine_noalloc(ctx, tar, sub)  # set-up on this device happens by now
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for s in range(5):
        tar, sub = landmark_set(30 + s, 100 + 700 * s)
        tw.fit_affine_noalloc(ctx, tar, sub)
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
