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
    """Free memory of the context's device is unchanged by the calls.  This
    reads the device-wide figure, so it assumes that no other process
    allocates on that GPU meanwhile (the test runs its calls back to back)."""
    tar, sub = landmark_set(7, 500)
    tw.fit_affine_noalloc(ctx, tar, sub)  # set-up on this device happens by now
    torch.cuda.synchronize(ctx.device)
    free0, _ = torch.cuda.mem_get_info(ctx.device)
    for s in range(5):
        tar, sub = landmark_set(30 + s, 100 + 700 * s)
        tw.fit_affine_noalloc(ctx, tar, sub)
    free1, _ = torch.cuda.mem_get_info(ctx.device)
    assert free1 == free0


def test_concurrent_callers_on_two_contexts_get_their_own_results(ctx):
    """Two contexts on one device share the scratch array; calls from two
    threads (ctypes releases the GIL during the call) must be serialised by
    the library so that each caller gets the matrix of its own landmarks."""
    import threading

    sets = [[landmark_set(100 + 10 * t + i, 64 + 97 * i) for i in range(12)] for t in range(2)]
    want = [[tw.fit_affine(ctx, tar, sub) for tar, sub in s] for s in sets]
    ctxs = [tw.Context(ctx.device), tw.Context(ctx.device)]
    got = [[None] * 12 for _ in range(2)]
    errors = []

    def run(t):
        try:
            for rep in range(3):
                for i, (tar, sub) in enumerate(sets[t]):
                    got[t][i] = tw.fit_affine_noalloc(ctxs[t], tar, sub)
                    np.testing.assert_allclose(got[t][i], want[t][i], rtol=0, atol=ATOL)
        except Exception as e:  # reported on the main thread
            errors.append(e)

    threads = [threading.Thread(target=run, args=(t,)) for t in range(2)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    for c in ctxs:
        c.close()
    assert not errors, errors[0]
