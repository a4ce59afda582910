"""The multi-rank host logic of bench.py on CPU: two gloo ranks reduce their
per-rank cells and times into the whole-job value (the cells every rank
advanced over the slowest rank's time), the way the NCCL ranks do on GPUs."""
import datetime
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=30))
    try:
        import bench
        mx, sm = bench._reducers(dist, "cpu")
        # rank r advanced 1000 (r + 1) cells for 10 loops in (r + 1) * 0.5 s
        mlups, t = bench.job_mlups(1000 * (rank + 1), 10, 0.5 * (rank + 1), mx, sm)
        q.put((rank, mlups, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_cells_over_slowest_time():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(ws))
    for _, mlups, t in res:
        assert t == pytest.approx(1.0)
        assert mlups == pytest.approx((1000 + 2000) * 10 / 1.0 / 1e6)


def test_single_rank_reducers_are_identity():
    sys.path.insert(0, ROOT)
    import bench
    mx, sm = bench._reducers(None, "cpu")
    assert bench.job_mlups(2_000_000, 100, 0.5, mx, sm) == (400.0, 0.5)
