"""The shared-memory staged TPS resample (TMA copies of each unit's source
footprint) against the gathering path and the FP64 oracle, and the bounded
waits of the kernels.

Both resample paths compute the same positions and end in the same
trilinear arithmetic, so their outputs must be identical bit for bit; the
oracle comparison uses the +-1 level criterion of the other parity tests.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import terawarp_b200 as tw
from oracle import oracle as O
from terawarp_b200 import synth

pytestmark = pytest.mark.gpu
TW_ERR_TIMEOUT = 5


def _hook(lib, name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


def _staging(ctx, on):
    f = _hook(ctx.lib, "tw_internal_set_resample_staging", C.c_int, [C.c_void_p, C.c_int])
    return f(ctx.handle, 1 if on else 0)


def _warp_both(ctx, vol, sub, tar, g):
    Z, Y, X = vol.shape
    t = tw.tps_solve(ctx, tar, sub)
    gsz = (tw.grid_size(X, g), tw.grid_size(Y, g), tw.grid_size(Z, g))
    nodes = tw.tps_eval_grid(ctx, t, gsz, g)
    t.close()
    outs = []
    for on in (1, 0):
        prev = _staging(ctx, on)
        try:
            dst = torch.empty_like(vol)
            tw.warp_tps_device(ctx, nodes, g, vol, dst)
            torch.cuda.synchronize()
            outs.append(dst)
        finally:
            _staging(ctx, prev)
    return outs, nodes


@pytest.mark.parametrize("g", [4, 8, 16, 32, 64])
@pytest.mark.parametrize("dtype", ["u8", "u16"])
def test_staged_equals_gathered_bit_for_bit(ctx, g, dtype):
    shape = (96, 160, 320)  # z, y, x: a few units per axis, partial units at the far x / y / z ends
    case = synth.large_tps_case(77 + g, "cuda", shape_zyx=shape, n=200, g=g, n_blobs=400, n_fibres=40)
    vol = case.vol if dtype == "u16" else (case.vol.to(torch.int32) >> 4).to(torch.uint8)
    (staged, gathered), _ = _warp_both(ctx, vol, case.marker_sub, case.marker_tar, g)
    assert torch.equal(staged, gathered)


def test_staged_large_job_matches_oracle_and_gather(ctx):
    shape = (256, 1024, 1024)
    case = synth.large_tps_case(1240, "cuda", shape_zyx=shape, n=1000, g=16)
    (staged, gathered), nodes = _warp_both(ctx, case.vol, case.marker_sub, case.marker_tar, 16)
    assert torch.equal(staged, gathered)
    # oracle on two 256^3 boxes, its own FP64 grid
    Z, Y, X = shape
    c, d = O.tps_solve(case.marker_tar, case.marker_sub)
    df = O.tps_grid(case.marker_tar, c, d, (O.grid_size(X, 16), O.grid_size(Y, 16), O.grid_size(Z, 16)), 16)
    src = case.vol.cpu().numpy()
    for (x0, y0, z0) in [(0, 0, 0), (512, 384, 0)]:
        ref = O.tps_warp_box(src, df, 16, (x0, y0, z0), (256, 256, 256))
        got = staged[z0:z0 + 256, y0:y0 + 256, x0:x0 + 256].cpu().numpy()
        dd = np.abs(got.astype(np.int64) - ref.astype(np.int64))
        assert (dd <= 1).mean() >= 0.9999, (x0, y0, z0, (dd <= 1).mean(), dd.max())


def test_solve_barrier_timeout_is_reported_and_context_recovers():
    """The cooperative solve's grid barrier gives up after its limit: with a
    1 us limit the CTAs that wait while CTA 0 factors the first diagonal
    block give up, every CTA returns, the call reports TW_ERR_TIMEOUT, and
    the same context then solves correctly with the default limit."""
    c = tw.Context(0)
    try:
        setlim = _hook(c.lib, "tw_internal_set_solve_barrier_ns", C.c_ulonglong, [C.c_void_p, C.c_ulonglong])
        rng = np.random.default_rng(5)
        sub = rng.uniform(5, 195, size=(300, 3)).astype(np.float32)
        tar = (sub + rng.normal(0, 2, size=sub.shape)).astype(np.float32)
        setlim(c.handle, 1000)
        with pytest.raises(tw.TeraWarpError) as e:
            tw.tps_solve(c, tar, sub)
        assert e.value.status == TW_ERR_TIMEOUT
        setlim(c.handle, 0)
        t = tw.tps_solve(c, tar, sub)
        cc, dd = t.coeffs()
        t.close()
        c0, d0 = O.tps_solve(tar, sub)
        np.testing.assert_allclose(cc, c0, atol=1e-7 * max(1.0, np.abs(c0).max()), rtol=0)
        np.testing.assert_allclose(dd, d0, atol=1e-7 * max(1.0, np.abs(d0).max()), rtol=0)
    finally:
        c.close()
