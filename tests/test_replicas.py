"""Replica bookkeeping of the multi-GPU bench path, run as two gloo ranks on
the CPU: barrier, max over ranks, per-rank seeds and the job value."""
import os

import pytest
import torch.multiprocessing as mp

from ezmock_b200.replicas import Replicas, job_seconds_per_mock, rank_seed


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    rep = Replicas(world, "gloo", timeout_s=60)
    try:
        rep.barrier()
        t = 1.5 + rank                       # this rank's device time
        tmax = rep.reduce_max(t)
        rep.barrier()
        q.put((rank, tmax, rank_seed(rank), job_seconds_per_mock(tmax, world, 10)))
    finally:
        rep.close()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.5, 2.5]          # max over ranks on every rank
    assert out[0][2] != out[1][2]                      # independent seeds
    assert out[0][3] == pytest.approx(2.5 / 20)        # s per mock for the whole job


def test_single_rank_needs_no_group():
    rep = Replicas(1)
    assert rep.dist is None
    assert rep.reduce_max(3.0) == 3.0
    rep.barrier()
    assert job_seconds_per_mock(2.0, 1, 4) == 0.5
