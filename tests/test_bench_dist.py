"""bench.py's multi-rank plumbing with two gloo ranks on the CPU: the
max-over-ranks timing reduction, the barrier, and the reference arm running
on rank 0 only (the other ranks return without work)."""

import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime

    import torch.distributed as dist
    bench = _bench()
    ws, r, local = bench.dist_setup()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        m = bench.allreduce_max(1.5 + r, ws)
        bench.barrier(ws)

        class A:
            warmup, steps, gpus, mg = 0, 1, world, 7

        called = []
        bench.oracle_solve = lambda mg: called.append(r) or (1.0, 27000, [0.0] * 32)
        bench.run_reference(A, ws, r)
        out.put((r, ws, local, m, called))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1]
    assert all(x[1] == 2 and x[3] == 2.5 for x in res)  # max over ranks
    assert res[0][4] == [0] and res[1][4] == []  # reference arm only on rank 0
