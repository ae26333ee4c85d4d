"""Serving: jobs of different sizes, types and landmark counts submitted
while others run; each result must be identical to the same job run alone,
and admission must respect the HBM budget."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import terawarp_b200 as tw
from oracle import oracle as O
from terawarp_b200 import api, synth

pytestmark = pytest.mark.gpu


def make_volume(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    hi = 256 if dtype == "u8" else 4096
    return rng.integers(0, hi, size=shape).astype(np.uint8 if dtype == "u8" else np.uint16)


def run_alone(ctx, spec, vol):
    if spec.kind == "tps":
        # values = ql_marker_tar, centres = ql_marker_sub
        return tw.imgwarp_smallmemory_image(ctx, spec.values, spec.centres, spec.g, spec.g, spec.g, 1, 0, vol)
    src = torch.from_numpy(vol).cuda()
    dst = torch.empty_like(src)
    tw.warp_affine_device(ctx, spec.M, src, dst)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


def test_batched_results_equal_alone_results(ctx):
    jobs = synth.serving_jobs(30, seed=77, dims_lo=(40, 36, 24), dims_hi=(200, 160, 64), n_lo=8, n_hi=300, g=8)
    vols = [make_volume(j.shape_zyx, j.dtype, i) for i, j in enumerate(jobs)]
    outs = [np.zeros_like(v) for v in vols]
    with api.Server(ctx, max_inflight=8) as srv:
        ids = []
        for j, v, o in zip(jobs, vols, outs):
            if j.kind == "tps":
                ids.append(srv.submit_tps(j.centres, j.values, j.g, v, o))
            else:
                ids.append(srv.submit_affine(j.M, v, o))
        lats = [srv.wait(i) for i in ids]
    assert all(l > 0 for l in lats)
    for j, v, o in zip(jobs, vols, outs):
        alone = run_alone(ctx, j, v)
        np.testing.assert_array_equal(o, alone, err_msg=f"{j.kind} {j.dtype} {j.shape_zyx}")


def test_served_tps_matches_oracle(ctx):
    jobs = [j for j in synth.serving_jobs(12, seed=5, dims_lo=(48, 40, 32), dims_hi=(96, 80, 48), n_lo=10, n_hi=60,
                                          g=8) if j.kind == "tps"][:3]
    with api.Server(ctx) as srv:
        for k, j in enumerate(jobs):
            v = make_volume(j.shape_zyx, j.dtype, 100 + k)
            o = np.zeros_like(v)
            srv.wait(srv.submit_tps(j.centres, j.values, j.g, v, o))
            ref = O.imgwarp_smallmemory_image(j.values, j.centres, j.g, v)
            d = np.abs(o.astype(np.int64) - ref.astype(np.int64))
            assert (d <= 1).mean() >= 0.9999


def test_admission_respects_hbm_budget(ctx):
    small = make_volume((16, 32, 32), "u8", 1)
    big = make_volume((64, 256, 256), "u16", 2)  # 8 MiB in + 8 MiB out
    M = np.eye(4)
    M[:3, 3] = [1.5, -2.0, 0.5]
    with api.Server(ctx, hbm_budget_bytes=4 << 20, max_inflight=4) as srv:
        o_big = np.zeros_like(big)
        o_small = np.zeros_like(small)
        jb = srv.submit_affine(M, big, o_big)
        js = srv.submit_affine(M, small, o_small)
        with pytest.raises(tw.TeraWarpError) as e:
            srv.wait(jb)
        assert e.value.status == 3  # TW_ERR_OOM: larger than the whole budget
        srv.wait(js)
    np.testing.assert_array_equal(o_small, O.affine_warp(small, M))


def test_many_small_jobs_complete(ctx):
    M = np.eye(4)
    M[:3, 3] = [0.25, 0.5, 0.75]
    vols = [make_volume((8 + i % 5, 20 + i % 7, 30 + i % 11), "u8" if i % 2 else "u16", i) for i in range(64)]
    outs = [np.zeros_like(v) for v in vols]
    with api.Server(ctx, max_inflight=16) as srv:
        ids = [srv.submit_affine(M, v, o) for v, o in zip(vols, outs)]
        for i in ids:
            srv.wait(i)
    for v, o in zip(vols, outs):
        np.testing.assert_array_equal(o, O.affine_warp(v, M))


def test_device_resident_jobs_equal_alone_results_and_report_stage_times(ctx):
    """Jobs whose volumes already live in HBM are warped in place (no copy);
    each result equals the job run alone, and every job reports its stage
    times in order."""
    jobs = synth.serving_jobs(24, seed=91, dims_lo=(64, 48, 32), dims_hi=(192, 160, 64), n_lo=8, n_hi=300, g=8)
    vols = [make_volume(j.shape_zyx, j.dtype, 200 + i) for i, j in enumerate(jobs)]
    d_src = [torch.from_numpy(v).cuda() for v in vols]
    d_out = [torch.empty_like(x) for x in d_src]
    with api.Server(ctx, max_inflight=8) as srv:
        ids = []
        for j, s, o in zip(jobs, d_src, d_out):
            if j.kind == "tps":
                ids.append(srv.submit_tps(j.centres, j.values, j.g, s, o))
            else:
                ids.append(srv.submit_affine(j.M, s, o))
        for i in ids:
            srv.wait(i)
        times = [srv.job_times(i) for i in ids]
    torch.cuda.synchronize()
    for j, v, o in zip(jobs, vols, d_out):
        np.testing.assert_array_equal(o.cpu().numpy(), run_alone(ctx, j, v), err_msg=f"{j.kind} {j.shape_zyx}")
    for j, t in zip(jobs, times):
        assert t["latency"] > 0 and t["queued"] >= 0
        assert t["ready"] is not None and t["resample_start"] is not None
        assert t["resample_end"] >= t["resample_start"] >= 0 and t["done"] >= t["resample_end"]
        if j.kind == "tps":
            assert t["solve"] is not None and t["grid"] >= t["solve"]
        else:
            assert t["solve"] is None and t["grid"] is None
