"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the
max-over-ranks timing and the status code every rank agrees on before any
raises (the N > 1 path runs independent replicas; these are its only
collectives)."""

import os
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path[:0] = [ROOT, os.path.join(ROOT, "dsa110-rt_b200")]
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
        code = bench.agreed_status(5 if rank == 1 else 0, world, "cpu")
        ok = bench.agreed_status(0, world, "cpu")
        out.put((rank, ms, code, ok))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_agreed_status_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert res == [(0, 15.0, 5, 0), (1, 15.0, 5, 0)]


def test_single_rank_needs_no_process_group():
    sys.path[:0] = [ROOT, os.path.join(ROOT, "dsa110-rt_b200")]
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.agreed_status(4, 1, "cpu") == 4
