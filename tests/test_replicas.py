"""Replica plumbing of bench.py on CPU: two gloo ranks, max-over-ranks timing
and the whole-job sum, as the GPU run uses them (the path does not shard, so
ranks exchange only these scalars)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    w, r, local, pg = bench.dist_setup(world)
    ms = 10.0 + 5.0 * r
    t = bench.max_over_ranks(pg, ms)
    total = bench.sum_over_ranks(pg, 1000.0 * (r + 1))
    bench.barrier(pg)
    q.put((r, w, t, total))
    pg.destroy_process_group()


def test_two_gloo_ranks_max_and_sum():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, t, total in out:
        assert w == 2
        assert t == 15.0          # max over ranks of 10 and 15 ms
        assert total == 3000.0    # 1000 + 2000 lattice updates


def test_reference_arm_other_ranks_exit_cleanly(monkeypatch):
    """Under torchrun only rank 0 of the reference arm does work."""
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("WORLD_SIZE", "1")
    monkeypatch.setenv("RANK", "0")
    w, r, local, pg = bench.dist_setup(1)
    assert (w, r, pg) == (1, 0, None)
