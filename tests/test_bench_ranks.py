"""The multi-rank path of bench.py (replicas, one process per GPU) on CPU:
two gloo ranks with different timings agree on the element-wise maximum,
and the whole-job throughput counts every rank's points over the slowest
rank's time."""
import importlib.util
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = _bench()
        mine = [10.0 + rank, 5.0 - rank, 2.5 * (rank + 1)]
        got = b.max_over_ranks(mine, dist, "cpu")
        out.put((rank, got, b.whole_job_points_per_s(world, 1 << 22, got[0])))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, got, value in res:
        assert got == [11.0, 5.0, 5.0]
        assert value == pytest.approx(2 * (1 << 22) / 11.0e-3)


def test_single_rank_passthrough():
    b = _bench()
    assert b.max_over_ranks([1.0, 2.0], None, "cpu") == [1.0, 2.0]
