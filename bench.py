"""Benchmark of the TPS warp hot path on B200.

Workload (one "step" = one whole TPS warp job): the large-TPS configuration,
a 2048 x 2048 x 1024 uint16 blob+fibre volume (8 GiB), 2000 landmark pairs on
a jittered lattice displaced by 8 random-phase sinusoids (amplitude <= 12) +
N(0, 1), B-spline control spacing 16, trilinear resampling: FP64 GPU solve,
FP32 compensated node evaluation, fused B-spline + trilinear resample.

  value   output GVoxel/s with the volume already in HBM (device-timed, CUDA
          events on the launching stream, max over ranks)
  e2e     the same job through the operator-level C ABI call with pinned host
          buffers (H2D of the volume and D2H of the result inside the timing)
  roofline  the resample kernel: algorithmic bytes (2 x 2 B per voxel + 12 B
          per node) / its measured duration vs MEASURED_PEAKS.json hbm_gbs
  cpu_baseline  the FP64 oracle (a restatement of the reference's CPU path)
          on the same inputs: solve and the whole node grid timed in full, the
          warp timed on the first 16-plane cell layer and scaled by the number
          of layers; all host threads, and (under "serial") one thread, the
          reference's own threading of the whole-image path
  accuracy  node displacement max / RMS against the FP64 oracle over the
          whole grid at spacing 8 and 16, and the share of output voxels
          within +-1 level on two 512^3 tiles of the measured output
  serving the serving mix (Poisson arrivals, mixed affine/rigid/TPS jobs of
          uneven sizes) through the continuous-batching server: p50/p99 job
          latency and aggregate GVoxel/s, capacity with every job submitted at
          once, and the plain one-job-at-a-time path on the same jobs

The volume (8 GiB) is far larger than L2 (126 MB), so no flush is needed
between iterations.  `--impl reference` times the reference's CPU path (the
oracle restatement; the reference itself cannot be built here) on the same
workload, metric and unit.  With torchrun (N > 1) every rank warps its own
replica (the path needs no collective); value = all ranks' voxels / max time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "TPS warp output GVoxel/s + HBM GB/s vs roofline; p50/p99 job latency"
SHAPE_ZYX = (1024, 2048, 2048)
N_LANDMARKS = 2000
G = 16
SEED = 1237
WORKLOAD = f"large_tps_{SHAPE_ZYX[2]}x{SHAPE_ZYX[1]}x{SHAPE_ZYX[0]}_u16_n{N_LANDMARKS}_g{G}"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-affine", action="store_true", help="skip the affine leg")
    ap.add_argument("--no-tiled", action="store_true", help="skip the tiled (out-of-core) leg")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the error figures against the FP64 oracle")
    ap.add_argument("--tb-layers", type=int, default=1, help="512-deep tile layers of the terabyte leg")
    ap.add_argument("--serve-jobs", type=int, default=1000, help="jobs in the serving leg")
    ap.add_argument("--small", action="store_true", help="256x256x128 case, 64 landmarks")
    ap.add_argument("--shape", type=str, default="", help="X,Y,Z volume for profiling captures (default: full)")
    ap.add_argument("--resample", choices=["staged", "gather"], default="staged",
                    help="TPS resample path: TMA-staged source footprint, or gathers from global memory")
    return ap.parse_args()


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling that covers the timed region.

    The sampler starts before the warm-up steps: nvidia-smi's own start-up
    (NVML initialisation) can stall the GPU for a moment, and that must not
    land inside the timed region.  mark_start() / mark_end() bracket the timed
    region; summary() keeps the samples taken inside it."""

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        self.t0 = self.t1 = None

    def __enter__(self):
        q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None
        return self

    def mark_start(self):
        self.t0 = datetime.datetime.now()

    def mark_end(self):
        self.t1 = datetime.datetime.now()

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.strip()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        parsed = []
        for r in rows:
            try:
                ts = datetime.datetime.strptime(r[0].strip(), "%Y/%m/%d %H:%M:%S.%f")
                parsed.append((ts, float(r[1].split()[0]), float(r[2].split()[0]),
                               [nm for nm, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v]))
            except (ValueError, IndexError):
                continue
        inside = parsed
        if self.t0 is not None and self.t1 is not None:
            pad = datetime.timedelta(seconds=0.25)
            inside = [x for x in parsed if self.t0 - pad <= x[0] <= self.t1 + pad] or parsed
        sm = [x[1] for x in inside]
        reasons = sorted({nm for x in inside for nm in x[3]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max((x[2] for x in inside), default=None),
                "reasons": reasons, "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=__import__("torch").device(f"cuda:{local}"))
    return ws, rank, local


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ----------------------------------------------------------------- CPU legs

SLAB_PLANES = G        # one whole cell layer: the oracle expands whole cells


def oracle_solve_grid(sub, tar, Z, threads):
    """FP64 oracle solve and whole node grid, each timed in full (their cost
    does not depend on the output planes).  Returns (c, d, grid, solve s, grid s,
    planes the first cell layer's samples can read)."""
    import numpy as np

    from oracle import oracle as O
    X, Y = SHAPE_ZYX[2], SHAPE_ZYX[1]
    t0 = time.perf_counter()
    c, d = O.tps_solve(tar, sub, 0.2, threads)
    t1 = time.perf_counter()
    gsz = (O.grid_size(X, G), O.grid_size(Y, G), O.grid_size(Z, G))
    df = O.tps_grid(tar, c, d, gsz, G, threads=threads)
    t2 = time.perf_counter()
    # the first cell layer's samples are convex combinations of node planes
    # 0..3 (B-spline weights >= 0, sum 1): q_z <= zmax, taps read planes up to
    # floor(zmax) + 1; two planes of margin on top
    zpos = (np.arange(4) - 1) * G
    zmax = float((df[:4, :, :, 2] + zpos[:, None, None]).max())
    need = int(min(Z, max(SLAB_PLANES, np.ceil(zmax) + 4)))
    return c, d, df, t1 - t0, t2 - t1, need


def cpu_slab_warp(planes, df, Z, threads, repeats=1):
    """Seconds of the oracle's warp of the first cell layer (SLAB_PLANES output
    planes, per-cell B-spline expansion included), median of `repeats`."""
    from oracle import oracle as O
    X, Y = SHAPE_ZYX[2], SHAPE_ZYX[1]
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        O.tps_warp_box(planes, df, G, (0, 0, 0), (X, Y, SLAB_PLANES), 0, threads, planes_of=Z)
        times.append(time.perf_counter() - t0)
    return statistics.median(times)


def cpu_baseline_figures(planes_fn, sub, tar, Z):
    """The FP64 oracle on the benchmark's own inputs, with the reference's
    whole-image threading (serial: no OpenMP in the grid loop or the block
    warp, q_imgwarp_tps_quicksmallmemory.cpp:620-648, :2121-2133) and with all
    host threads (OpenMP).  Solve and node grid are timed in full; the warp is
    timed on the first cell layer and scaled by Z / SLAB_PLANES (its cost is
    the same per cell layer).  planes_fn(k) returns the volume's first k
    planes as a (k, Y, X) array."""
    from oracle import oracle as O
    X, Y = SHAPE_ZYX[2], SHAPE_ZYX[1]
    out = {}
    planes = None
    for label, threads in (("omp", O.max_threads()), ("serial", 1)):
        c, d, df, ts, tg, need = oracle_solve_grid(sub, tar, Z, threads)
        if planes is None or planes.shape[0] < need:
            planes = planes_fn(need)
        slab = cpu_slab_warp(planes, df, Z, threads)
        job = ts + tg + slab * (Z / SLAB_PLANES)
        out[label] = {"value": X * Y * Z / job / 1e9, "threads": threads, "job_s": job, "solve_s": ts,
                      "grid_s": tg, "slab_warp_s": slab}
    return out


def cpu_sample_text(fig):
    return (f"FP64 oracle (restatement of the reference CPU path) on the benchmark's own inputs: solve "
            f"(n={N_LANDMARKS}) and the whole g={G} node grid timed in full; warp timed on the first "
            f"{SLAB_PLANES}-plane cell layer of the {SHAPE_ZYX[2]}x{SHAPE_ZYX[1]} volume and scaled by "
            f"{SHAPE_ZYX[0] // SLAB_PLANES} layers; {fig['threads']} thread(s)")


def run_reference(args):
    """The reference arm: the FP64 oracle restatement of the reference's CPU
    path on all host threads, on the same workload and inputs as our arm
    (landmarks and volume planes from the same seed).  Solve and node grid are
    timed once in full; each step warps the first cell layer; the job time is
    solve + grid + layers x median layer time.  Rank 0 alone runs it."""
    ws, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from terawarp_b200 import synth
    threads = O.max_threads()
    Z, Y, X = SHAPE_ZYX
    lm = synth.large_tps_case(SEED, "cpu", shape_zyx=SHAPE_ZYX, n=N_LANDMARKS, g=G, z_range=(0, 1))
    sub, tar = lm.marker_sub, lm.marker_tar
    if args.warmup > 0:
        oracle_solve_grid(sub, tar, Z, threads)
    c, d, df, ts, tg, need = oracle_solve_grid(sub, tar, Z, threads)
    planes = synth.large_tps_case(SEED, "cpu", shape_zyx=SHAPE_ZYX, n=N_LANDMARKS, g=G,
                                  z_range=(0, need)).vol.numpy()
    for _ in range(args.warmup):
        cpu_slab_warp(planes, df, Z, threads)
    slabs = [cpu_slab_warp(planes, df, Z, threads) for _ in range(args.steps)]
    job = ts + tg + statistics.median(slabs) * (Z / SLAB_PLANES)
    v = X * Y * Z / job / 1e9
    fig = {"threads": threads}
    line = {"metric": METRIC, "value": v, "unit": "GVoxel/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": job * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "volume_xyz": [X, Y, Z], "landmarks": N_LANDMARKS, "grid_spacing": G,
                       "interp": "trilinear"},
            "cpu_baseline": {"value": v, "unit": "GVoxel/s", "cores": threads, "kind": "port",
                             "sample": cpu_sample_text(fig), "solve_s": ts, "grid_s": tg,
                             "slab_warp_s": [round(x, 4) for x in slabs]},
            "e2e": {"value": v, "unit": "GVoxel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------- other legs

def affine_leg(ctx, device: int, steps: int = 5):
    """The affine configuration: a 1024 x 1024 x 512 uint16 blob+fibre volume
    warped by the 12-parameter affine fitted from 32 landmark pairs, device
    resident; CUDA-event time per warp and its HBM roofline (2 x 2 B per
    output voxel)."""
    import torch

    import terawarp_b200 as tw
    from terawarp_b200 import synth

    case = synth.affine_case(device=f"cuda:{device}")
    src = case.vol
    dst = torch.empty_like(src)
    M = tw.fit_affine(ctx, case.marker_tar, case.marker_sub)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(3):
        tw.warp_affine_device(ctx, M, src, dst, 0, stream=stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(steps):
        tw.warp_affine_device(ctx, M, src, dst, 0, stream=stream)
    ev[1].record()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / steps
    vox = src.numel()
    peak, _ = measured_peaks()
    gbs = vox * 4 / (ms / 1e3) / 1e9
    del src, dst
    return {"workload": "affine_1024x1024x512_u16_n32", "ms_per_warp": ms, "gvoxel_s": vox / (ms / 1e3) / 1e9,
            "achieved_gbs": gbs, "frac_of_hbm": gbs / peak, "kernel": "k_resample_affine<uint16,trilinear>"}


def tiled_leg(ctx, device: int, shape_zyx=(512, 2048, 2048)):
    """The out-of-core TPS path: a 2048 x 2048 x 512 uint16 volume in pinned
    host memory (2000 landmarks, g = 16) warped tile by tile (source boxes =
    the tiles' exact sample footprints) with the tile shape and staging depth
    the autotuner picks on the volume's corner block: solve, node grid, reads,
    H2D, kernels, D2H and writes all inside the wall-clock time."""
    import torch

    from terawarp_b200 import api, autotune, synth

    Z, Y, X = shape_zyx
    vol = synth.blob_volume(shape_zyx, "u16", SEED + 11, n_blobs=5000, n_fibres=1000, device=f"cuda:{device}")
    h_src = torch.empty(shape_zyx, dtype=torch.uint16, pin_memory=True)
    h_src.copy_(vol)
    del vol
    h_out = torch.empty(shape_zyx, dtype=torch.uint16, pin_memory=True)
    sub, tar = synth.lattice_landmarks((X, Y, Z), N_LANDMARKS, SEED + 12)
    # reference argument order: (ql_marker_tar = values, ql_marker_sub = centres)
    tile, depth, table = autotune.tune_tiled_tps(ctx, sub, tar, 1.0, G, h_src)
    api.imgwarp_smallmemory_tiled(ctx, sub, tar, 1.0, G, h_src, out=h_out, tile=tile, depth=depth)  # warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    api.imgwarp_smallmemory_tiled(ctx, sub, tar, 1.0, G, h_src, out=h_out, tile=tile, depth=depth)
    torch.cuda.synchronize()
    s = time.perf_counter() - t0
    vox = X * Y * Z
    del h_src, h_out
    return {"workload": f"tiled_tps_{X}x{Y}x{Z}_u16_n{N_LANDMARKS}_g{G}", "tile_xyz": list(tile),
            "staging_depth": depth, "seconds": s, "gvoxel_s": vox / s / 1e9,
            "autotune": [{"tile_xyz": list(t), "depth": d, "sample_s": round(x, 4)} for t, d, x in table],
            "path": "tw_imgwarp_smallmemory_tiled, pinned host volumes (built-in box reader/writer)"}


def copy_peaks(device: int, nbytes: int = 1 << 30):
    """Measured pinned host <-> HBM copy bandwidth (GB/s): H2D alone, D2H
    alone, and both directions at once (the tiled path's steady state)."""
    import torch
    h_a = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    h_b = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d_a = torch.empty(nbytes, dtype=torch.uint8, device=f"cuda:{device}")
    d_b = torch.empty(nbytes, dtype=torch.uint8, device=f"cuda:{device}")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    out = {}
    for name, ops in (("h2d", [(s1, d_a, h_a)]), ("d2h", [(s1, h_a, d_a)]),
                      ("both", [(s1, d_a, h_a), (s2, h_b, d_b)])):
        for rep in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for st, dst, src in ops:
                with torch.cuda.stream(st):
                    dst.copy_(src, non_blocking=True)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
        out[name + "_gbs"] = len(ops) * nbytes / dt / 1e9
    del h_a, h_b, d_a, d_b
    return out


def terabyte_leg(ctx, device: int, layers: int = 1):
    """The terabyte tiled configuration at its stated geometry: a 16384 x 16384
    x 4096 uint16 volume generated procedurally per 512^3 tile from a seeded
    hash (no stored volume), 4096 landmark pairs with the sinusoidal
    displacement model, g = 16, warped tile by tile (512^3 tiles, three in
    flight) for `layers` 512-deep tile layers into a checksum sink.  Reports
    output GVoxel/s, the host-link bytes and their fraction of the measured
    pinned-copy bandwidth (both directions at once), and the FP64 solve and
    whole node-grid times at N = 4096."""
    import numpy as np
    import torch

    import terawarp_b200 as tw
    from terawarp_b200 import api, synth

    Z, Y, X = 4096, 16384, 16384
    n, g = 4096, 16
    sub, tar = synth.lattice_landmarks((X, Y, Z), n, SEED + 21)
    # solve and the whole node grid at N = 4096, each timed on its own
    gsz = (tw.grid_size(X, g), tw.grid_size(Y, g), tw.grid_size(Z, g))
    t = tw.tps_solve(ctx, tar, sub)
    nodes = tw.tps_eval_grid(ctx, t, gsz, g)
    t.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t = tw.tps_solve(ctx, tar, sub)
    solve_s = time.perf_counter() - t0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    stream = torch.cuda.current_stream().cuda_stream
    ev[0].record()
    tw.tps_eval_grid(ctx, t, gsz, g, out=nodes, stream=stream)
    ev[1].record()
    torch.cuda.synchronize()
    grid_ms = ev[0].elapsed_time(ev[1])
    t.close()
    del nodes
    torch.cuda.empty_cache()
    peaks = copy_peaks(device)
    src = api.SyntheticVolume((Z, Y, X), np.uint16, seed=SEED + 22)
    region = ((0, 0, 0), (X, Y, 512 * layers))
    # warm-up on a corner (kernels, pinned slots, the base block)
    api.imgwarp_smallmemory_tiled(ctx, sub, tar, 1.0, g, src, out=api.Checksum(np.uint16), tile=(512, 512, 512),
                                  depth=3, region=((0, 0, 0), (1024, 1024, 512)))
    sink = api.Checksum(np.uint16)
    torch.cuda.synchronize()
    b0 = ctx.transfer_bytes
    t0 = time.perf_counter()
    api.imgwarp_smallmemory_tiled(ctx, sub, tar, 1.0, g, src, out=sink, tile=(512, 512, 512), depth=3, region=region)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    b1 = ctx.transfer_bytes
    h2d, d2h = b1[0] - b0[0], b1[1] - b0[1]
    vox = X * Y * 512 * layers
    _, _, got = sink.value
    return {"workload": f"tiled_tps_{X}x{Y}x{Z}_u16_n{n}_g{g}", "region_z": [0, 512 * layers],
            "tiles": (X // 512) * (Y // 512) * layers, "voxels": vox, "sink_voxels": got,
            "seconds": wall, "gvoxel_s": vox / wall / 1e9,
            "h2d_bytes": h2d, "d2h_bytes": d2h, "h2d_gbs": h2d / wall / 1e9, "d2h_gbs": d2h / wall / 1e9,
            "copy_peaks": peaks, "link_frac_of_bidirectional_peak": (h2d + d2h) / wall / 1e9 / peaks["both_gbs"],
            "solve_n4096_s": solve_s, "node_grid_ms": grid_ms, "node_grid_nodes": gsz[0] * gsz[1] * gsz[2],
            "note": "solve + whole node grid + tile reads, H2D, kernels, D2H and sink inside the wall time; "
                    "procedural source (seeded-hash base block shifted per 512^3 tile), checksum sink"}


# ------------------------------------------------------------- serving leg

class _RingAlloc:
    """Recycled output buffers: slices of one preallocated buffer handed out in
    submission order; a slice is reused once the job that held it finished
    (wait(job) is called for jobs whose slice would be overwritten)."""

    def __init__(self, nbytes: int, wait):
        self.n, self.head, self.live, self.wait = nbytes, 0, [], wait

    def take(self, nbytes: int, job_key) -> int:
        if nbytes > self.n:
            raise ValueError("job larger than the output ring")
        # slices start on 256-byte boundaries (any voxel type, aligned DMA)
        head = (self.head + 255) & ~255
        start = head if head + nbytes <= self.n else 0
        end = start + nbytes
        keep = []
        for (k, a, b) in self.live:
            if a < end and start < b:
                self.wait(k)
            else:
                keep.append((k, a, b))
        self.live = keep + [(job_key, start, end)]
        self.head = end
        return start


def serving_leg(ctx, device: int, n_jobs: int, seed: int = 1239, rate_hz: float = 20.0):
    """The serving mix (Poisson arrivals at rate_hz, dims log-uniform 128^3 ..
    1024x1024x256, u8/u16, 30% affine / 10% rigid / 60% TPS with 16-4096
    landmarks) through the continuous-batching server.

    host: volumes in pinned host memory (outputs in a recycled pinned ring):
      p50/p99 job latency (submit -> result in host memory) under Poisson
      arrivals, aggregate GVoxel/s, capacity with every job submitted at once,
      and the plain one-job-at-a-time path (one operator-level call per job,
      H2D and D2H included) on the same jobs.
    device: the same jobs with volumes already in HBM (outputs in a recycled
      device ring): capacity of the server against the plain one-job-at-a-time
      GPU path (solve, node grid and warp per job, each waited for).
    Stage times (queue wait, solve, resample) come from tw_server_job_times."""
    import numpy as np
    import torch

    import terawarp_b200 as tw
    from terawarp_b200 import api, synth

    dev = f"cuda:{device}"
    jobs = synth.serving_jobs(n_jobs, seed=seed, rate_hz=rate_hz)
    tdt = {"u8": torch.uint8, "u16": torch.uint16}
    esz = {"u8": 1, "u16": 2}
    nbytes = [int(np.prod(j.shape_zyx)) * esz[j.dtype] for j in jobs]
    vox = sum(int(np.prod(j.shape_zyx)) for j in jobs)
    big = max(nbytes)
    # inputs: views of one pool of random bytes (jobs only read them)
    h_pool = torch.empty(big, dtype=torch.uint8, pin_memory=True)
    h_pool.copy_(torch.randint(0, 256, (big,), dtype=torch.uint8, device=dev))
    d_pool = h_pool.to(dev)
    ring_bytes = max(4 * big, 4 << 30)
    h_ring = torch.empty(ring_bytes, dtype=torch.uint8, pin_memory=True)
    d_ring = torch.empty(ring_bytes, dtype=torch.uint8, device=dev)

    def view(pool, off, j, b):
        return pool[off:off + b].view(tdt[j.dtype]).reshape(j.shape_zyx)

    def submit(srv, j, src, dst):
        if j.kind == "tps":
            return srv.submit_tps(j.centres, j.values, j.g, src, dst)
        return srv.submit_affine(j.M, src, dst)

    def served(srv, pool, ring_pool, poisson: bool):
        ids = {}
        ring = _RingAlloc(ring_bytes, lambda k: srv.wait(ids[k]))
        t0 = time.perf_counter()
        for i, (j, b) in enumerate(zip(jobs, nbytes)):
            if poisson:
                delay = t0 + j.arrival_s - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
            off = ring.take(b, i)
            ids[i] = submit(srv, j, view(pool, 0, j, b), view(ring_pool, off, j, b))
        lats = [srv.wait(ids[i]) for i in range(len(jobs))]
        wall = time.perf_counter() - t0
        times = [srv.job_times(ids[i]) for i in range(len(jobs))]
        return wall, lats, times

    def pct(v, q):
        v = [x for x in v if x is not None]
        return float(np.percentile(v, q)) * 1e3 if v else None

    def stage_summary(times):
        solve = [t["solve"] for t in times]
        rs = [None if t["resample_start"] is None else t["resample_end"] - t["resample_start"] for t in times]
        queued = [t["queued"] for t in times]
        return {"queued_p50_ms": pct(queued, 50), "queued_p99_ms": pct(queued, 99),
                "solve_done_p50_ms": pct(solve, 50), "resample_round_p50_ms": pct(rs, 50),
                "resample_round_p99_ms": pct(rs, 99)}

    def plain_host(j, src, dst):
        if j.kind == "tps":
            tw.imgwarp_smallmemory_image(ctx, j.values, j.centres, j.g, j.g, j.g, 1, 0, src, out=dst)
        else:
            d_src = src.to(dev, non_blocking=True)
            d_dst = torch.empty_like(d_src)
            tw.warp_affine_device(ctx, j.M, d_src, d_dst)
            dst.copy_(d_dst)
        torch.cuda.synchronize()

    def plain_device(j, src, dst):
        if j.kind == "tps":
            Z, Y, X = j.shape_zyx
            t = tw.tps_solve(ctx, j.centres, j.values)
            nodes = tw.tps_eval_grid(ctx, t, (tw.grid_size(X, j.g), tw.grid_size(Y, j.g), tw.grid_size(Z, j.g)), j.g)
            tw.warp_tps_device(ctx, nodes, j.g, src, dst)
            t.close()
        else:
            tw.warp_affine_device(ctx, j.M, src, dst)
        torch.cuda.synchronize()

    def sequential(plain, pool, ring_pool):
        for i in range(min(4, len(jobs))):  # warm
            plain(jobs[i], view(pool, 0, jobs[i], nbytes[i]), view(ring_pool, 0, jobs[i], nbytes[i]))
        t0 = time.perf_counter()
        off = 0
        for j, b in zip(jobs, nbytes):
            off = 0 if off + b > ring_bytes else off
            plain(j, view(pool, 0, j, b), view(ring_pool, off, j, b))
            off = (off + b + 255) & ~255  # 256-byte aligned slices (any voxel type)
        return time.perf_counter() - t0

    out = {"jobs": n_jobs, "rate_hz": rate_hz,
           "mix": {k: sum(1 for j in jobs if j.kind == k) for k in ("affine", "rigid", "tps")}, "voxels": vox}
    with api.Server(ctx) as srv:
        served(srv, h_pool, h_ring, False)  # untimed: grows the pools, loads every kernel variant
        wall_p, lats, times_p = served(srv, h_pool, h_ring, True)
        wall_s, _, times_s = served(srv, h_pool, h_ring, False)
    t_seq = sequential(plain_host, h_pool, h_ring)
    lat_ms = sorted(1e3 * v for v in lats)
    out["host"] = {
        "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
        "poisson_gvoxel_s": vox / wall_p / 1e9, "poisson_wall_s": wall_p,
        "saturated_gvoxel_s": vox / wall_s / 1e9, "sequential_gvoxel_s": vox / t_seq / 1e9,
        "saturated_over_sequential": t_seq / wall_s,
        "stages_poisson": stage_summary(times_p), "stages_saturated": stage_summary(times_s),
        "path": "tw_server_* from pinned host buffers (recycled output ring) vs one operator-level call per job"}
    with api.Server(ctx) as srv:
        served(srv, d_pool, d_ring, False)
        wall_d, lats_d, times_d = served(srv, d_pool, d_ring, False)
    t_seq_d = sequential(plain_device, d_pool, d_ring)
    lat_d = sorted(1e3 * v for v in lats_d)
    out["device"] = {
        "saturated_gvoxel_s": vox / wall_d / 1e9, "sequential_gvoxel_s": vox / t_seq_d / 1e9,
        "saturated_over_sequential": t_seq_d / wall_d,
        "saturated_p50_ms": float(np.percentile(lat_d, 50)), "saturated_p99_ms": float(np.percentile(lat_d, 99)),
        "stages": stage_summary(times_d),
        "path": "tw_server_* on device-resident volumes vs solve + node grid + warp per job, each waited for"}
    del h_pool, d_pool, h_ring, d_ring
    return out


# ----------------------------------------------------------- accuracy

def accuracy_leg(ctx, case, dst, tile: int = 512):
    """Errors of the benchmark job against the FP64 oracle: node displacement
    max / RMS (voxels) over the whole control grid at spacing 8 and 16, and
    the share of output voxels within +-1 level (and exact) on two tile^3
    boxes -- the corner tile and a seeded interior one -- of the measured
    g = 16 output `dst`, the oracle using its own FP64 solve and node grid."""
    import numpy as np
    import torch

    import terawarp_b200 as tw
    from oracle import oracle as O

    Z, Y, X = case.vol.shape
    tar, sub = case.marker_tar, case.marker_sub
    c, d = O.tps_solve(tar, sub)
    out = {}
    for g in (8, 16):
        gsz = (tw.grid_size(X, g), tw.grid_size(Y, g), tw.grid_size(Z, g))
        t = tw.tps_solve(ctx, tar, sub)
        nodes = tw.tps_eval_grid(ctx, t, gsz, g)
        torch.cuda.synchronize()
        t.close()
        ref = O.tps_grid(tar, c, d, gsz, g)
        err = np.abs(nodes[..., :3].cpu().numpy().astype(np.float64) - ref.astype(np.float64))
        del nodes
        out[f"g{g}"] = {"nodes": int(err.size // 3), "node_max_err_vox": float(err.max()),
                        "node_rms_err_vox": float(np.sqrt((err ** 2).mean()))}
        if g != 16:
            continue
        src_h = case.vol.cpu().numpy()
        rng = np.random.default_rng(2024)
        t = min(tile, X, Y, Z)
        boxes = [(0, 0, 0), tuple(int(v) for v in rng.integers(0, [X - t + 1, Y - t + 1, Z - t + 1]))]
        n_in = n_ex = n = 0
        dmax = 0
        for (x0, y0, z0) in boxes:
            r = O.tps_warp_box(src_h, ref, g, (x0, y0, z0), (t, t, t))
            got = dst[z0:z0 + t, y0:y0 + t, x0:x0 + t].cpu().numpy()
            dd = np.abs(got.astype(np.int64) - r.astype(np.int64))
            n_in += int((dd <= 1).sum())
            n_ex += int((dd == 0).sum())
            n += dd.size
            dmax = max(dmax, int(dd.max()))
        del src_h
        out["intensity_g16"] = {"within1_frac": n_in / n, "exact_frac": n_ex / n, "max_diff": dmax, "voxels": n,
                                "boxes_xyz": [list(b) for b in boxes], "box_edge": t}
    out["reference"] = "FP64 oracle: solve, node grid (stored as float) and per-cell B-spline warp in double"
    return out


# ----------------------------------------------------------------- our arm

def run_ours(args):
    import numpy as np
    import torch

    import terawarp_b200 as tw
    from terawarp_b200 import synth

    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    shape = (128, 256, 256) if args.small else SHAPE_ZYX
    if args.shape:
        sx, sy, sz = (int(v) for v in args.shape.split(","))
        shape = (sz, sy, sx)
    Z, Y, X = shape
    n = 64 if args.small else N_LANDMARKS
    case = synth.large_tps_case(SEED + rank, dev, shape_zyx=shape, n=n, g=G)
    src = case.vol
    dst = torch.empty_like(src)
    sub, tar = case.marker_sub, case.marker_tar
    ctx = tw.Context(local)
    if args.resample == "gather":
        set_staging = ctx.lib.tw_internal_set_resample_staging
        set_staging.restype, set_staging.argtypes = C.c_int, [C.c_void_p, C.c_int]
        set_staging(ctx.handle, 0)
    gsz = (tw.grid_size(X, G), tw.grid_size(Y, G), tw.grid_size(Z, G))
    nodes = torch.empty((gsz[2], gsz[1], gsz[0], 4), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream

    def step(ev=None):
        t = tw.tps_solve(ctx, tar, sub)                 # FP64 solve (centres = target markers)
        if ev is not None:
            ev[0].record()
        tw.tps_eval_grid(ctx, t, gsz, G, out=nodes, stream=stream)
        if ev is not None:
            ev[1].record()
        tw.warp_tps_device(ctx, nodes, G, src, dst, 0, stream=stream)
        if ev is not None:
            ev[2].record()
        return t

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    keep = []
    with Clocks(local) as clk:
        t_warm = time.perf_counter()
        for _ in range(args.warmup):
            step().close()
        torch.cuda.synchronize()
        # warm-up lasts at least 2 s so that the sampler's start-up is over
        while time.perf_counter() - t_warm < 2.0:
            step().close()
            torch.cuda.synchronize()
        launches0 = ctx.kernel_launches
        barrier(ws)
        torch.cuda.synchronize()
        clk.mark_start()
        for i in range(args.steps):
            evs[i][3].record()
            keep.append(step(evs[i][:3]))
        torch.cuda.synchronize()
        barrier(ws)
        clk.mark_end()
    launches = ctx.kernel_launches - launches0
    for t in keep:
        t.close()
    step_ms = [evs[i][3].elapsed_time(evs[i][2]) for i in range(args.steps)]
    solve_ms = [evs[i][3].elapsed_time(evs[i][0]) for i in range(args.steps)]
    eval_ms = [evs[i][0].elapsed_time(evs[i][1]) for i in range(args.steps)]
    warp_ms = [evs[i][1].elapsed_time(evs[i][2]) for i in range(args.steps)]
    total_ms = max_over_ranks(sum(step_ms), ws)
    vox = X * Y * Z
    value = ws * vox * args.steps / (total_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    alg_bytes = vox * 2 * 2 + 12 * gsz[0] * gsz[1] * gsz[2]
    warp_avg = statistics.mean(warp_ms)
    achieved = alg_bytes / (warp_avg / 1e3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / "traffic.json"
    if prof.exists():
        try:
            traffic = json.loads(prof.read_text()).get(WORKLOAD if not args.small else "small")
        except Exception:
            traffic = None
    pairs = gsz[0] * gsz[1] * gsz[2] * n
    eval_avg = statistics.mean(eval_ms)
    clocks = clk.summary()
    fp32_peak_tflops = 148 * 128 * 2 * (clocks["sm_mhz"] or 1965.0) * 1e6 / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": "GVoxel/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16",
        "data": "synthetic: seeded blob+fibre uint16 volume, jittered-lattice landmarks with sinusoidal displacement",
        "config": {"workload": (WORKLOAD if not (args.small or args.shape)
                                else f"tps_{X}x{Y}x{Z}_u16_n{n}_g{G}"),
                   "volume_xyz": [X, Y, Z], "landmarks": n, "grid_spacing": G, "interp": "trilinear",
                   "parallelism": f"replicas x{ws}", "l2": "input 8 GiB > 126 MB L2 (no flush needed)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind, "kernel": ("k_tps_plan + k_tps_lists + k_tps_staged x2 + k_tps_gather<uint16,16>" if args.resample == "staged"
                                else "k_tps_gather<uint16,16>"),
                     "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": warp_avg},
        "gpu_launches": launches,
        "clocks": clocks,
        "stages_ms": {"solve_fp64": statistics.mean(solve_ms), "node_eval_fp32": eval_avg, "resample": warp_avg},
        "resample_ms_per_step": [round(v, 3) for v in warp_ms],
        "solve_ms_per_step": [round(v, 3) for v in solve_ms],
        "tps_eval": {"pairs": pairs, "flop_per_pair": 15, "tflops": pairs * 15 / (eval_avg / 1e3) / 1e12,
                     "fp32_peak_tflops_at_clock": fp32_peak_tflops,
                     "frac": pairs * 15 / (eval_avg / 1e3) / 1e12 / fp32_peak_tflops},
    }
    # e2e: operator-level call with pinned host buffers
    if not args.no_e2e:
        h_src = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
        h_src.copy_(src)
        h_dst = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
        torch.cuda.synchronize()
        tw.imgwarp_smallmemory_image(ctx, sub, tar, G, G, G, 1, 0, h_src, out=h_dst)  # warm
        times = []
        for _ in range(max(1, min(args.steps, 3))):
            barrier(ws)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tw.imgwarp_smallmemory_image(ctx, sub, tar, G, G, G, 1, 0, h_src, out=h_dst)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(statistics.mean(times), ws)
        line["e2e"] = {"value": ws * vox / e2e_s / 1e9, "unit": "GVoxel/s", "h2d_bytes_per_step": vox * 2,
                       "d2h_bytes_per_step": vox * 2, "path": "tw_imgwarp_smallmemory_image, pinned host buffers",
                       "ms_per_step": e2e_s * 1e3}
        equal = bool(torch.equal(h_dst, dst.cpu()))
        line["e2e"]["matches_device_path"] = equal
        # the host link bounds e2e: its bytes per step over the measured
        # rate of pinned copies in both directions at once on this box
        link = copy_peaks(local)
        link_gbs = 2 * vox * 2 / e2e_s / 1e9
        line["e2e"]["link"] = {"achieved_gbs": link_gbs, "both_directions_peak_gbs": link["both_gbs"],
                               "frac": link_gbs / link["both_gbs"], "h2d_peak_gbs": link["h2d_gbs"],
                               "d2h_peak_gbs": link["d2h_gbs"]}
        del h_src, h_dst
    if rank == 0 and not args.no_accuracy:
        line["accuracy"] = accuracy_leg(ctx, case, dst)
    if rank == 0 and not args.no_affine and not args.small and not args.shape:
        line["affine"] = affine_leg(ctx, local)
    if rank == 0 and not args.no_tiled and not args.small and not args.shape:
        line["tiled"] = tiled_leg(ctx, local)
        line["terabyte"] = terabyte_leg(ctx, local, args.tb_layers)
    if rank == 0 and not args.no_serve and not args.small and not args.shape:
        line["serving"] = serving_leg(ctx, local, args.serve_jobs)
    if rank == 0 and ws == 1 and not args.no_cpu and not args.small and not args.shape:
        figs = cpu_baseline_figures(lambda k: src[:k].cpu().numpy(), sub, tar, Z)
        omp, ser = figs["omp"], figs["serial"]
        line["cpu_baseline"] = {"value": omp["value"], "unit": "GVoxel/s", "cores": omp["threads"], "kind": "port",
                                "sample": cpu_sample_text(omp), "solve_s": omp["solve_s"], "grid_s": omp["grid_s"],
                                "slab_warp_s": omp["slab_warp_s"],
                                "serial": {"value": ser["value"], "unit": "GVoxel/s", "cores": 1,
                                           "sample": cpu_sample_text(ser), "solve_s": ser["solve_s"],
                                           "grid_s": ser["grid_s"], "slab_warp_s": ser["slab_warp_s"]}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
