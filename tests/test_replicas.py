"""The multi-GPU path is replicas only: every rank warps its own job and the
bench reports all ranks' voxels over the slowest rank's time.  These CPU tests
run that host logic as two gloo ranks."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, ws: int, port: int, times, q):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        bench.barrier(ws)
        t = bench.max_over_ranks(times[rank], ws)
        bench.barrier(ws)
        q.put((rank, t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_aggregate_value():
    ws, port = 2, _free_port()
    times = [1.25, 2.5]  # seconds per rank for the same per-rank work
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, times, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(ws))
    assert got == {0: 2.5, 1: 2.5}  # every rank sees the slowest rank's time
    # value = all ranks' units / the slowest time (weak scaling)
    vox, steps = 1000, 4
    assert ws * vox * steps / got[0] == pytest.approx(3200.0)
