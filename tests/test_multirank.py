"""The multi-rank path of bench.py on the CPU: two gloo ranks, as torchrun
launches them (RANK / WORLD_SIZE / LOCAL_RANK, rendezvous on 127.0.0.1),
each timing its own replica; every rank reports the largest per-step time
and the whole-job value counts the positions of all ranks (weak scaling,
no collective on the data path)."""
from __future__ import annotations

import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist

    import bench

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    r, w, local = bench.dist_env()
    dist.init_process_group("gloo", rank=r, world_size=w)
    try:
        ms = 10.0 + 5.0 * r          # this rank's replica time
        worst = bench.max_over_ranks(ms, w, device="cpu")
        positions = 1000             # per replica
        q.put((r, local, worst, positions * w / (worst / 1e3)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[0] for g in got] == [0, 1] and [g[1] for g in got] == [0, 1]
    assert all(g[2] == 15.0 for g in got)
    assert all(abs(g[3] - 2000 / 0.015) < 1e-6 for g in got)


def test_one_rank_is_unchanged():
    import bench

    assert bench.max_over_ranks(12.5, 1) == 12.5
