"""Replica plumbing with two gloo ranks on the CPU (the multi-GPU path's host logic).

Each rank times its own box; the job's time is the maximum over ranks and the
throughput is world x units / that maximum.  Ranks are spawned processes
rendezvousing on 127.0.0.1.
"""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(world))
    from ifdm_code_b200.replicas import Replicas

    r = Replicas("gloo", timeout_s=60)
    r.barrier()
    t = 1.0 + rank  # rank 1 is the slow one
    tmax = r.max(t)
    out[rank] = (tmax, r.throughput(1000.0, tmax), r.world)
    r.barrier()
    r.close()


def test_two_gloo_ranks_take_the_max_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        tmax, thr, w = out[r]
        assert tmax == pytest.approx(2.0) and w == 2
        assert thr == pytest.approx(2 * 1000.0 / 2.0)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from ifdm_code_b200.replicas import Replicas

    r = Replicas("gloo")
    assert r.world == 1 and r.max(3.5) == 3.5 and r.throughput(10.0, 2.0) == 5.0
    r.barrier()
    r.close()
