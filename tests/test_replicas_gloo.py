"""CPU tests of the multi-GPU replica logic with a world_size-2 gloo
process group: ranks render disjoint orbit frames, the timing reduction is
the max over ranks, and the whole-job rate counts every rank's frames."""
from __future__ import annotations

import os

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from gamesplat_b200 import replicas


def _worker(rank, world, port, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        frames = replicas.frames_for_rank(rank, world, 5, 12, 120)
        t = 1.0 + rank            # rank 1 is the slow one
        tmax = replicas.reduce_max(t, dist)
        gathered = [None] * world
        dist.all_gather_object(gathered, frames)
        results[rank] = (frames, tmax, gathered)
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_over_gloo():
    world = 2
    port = 29500 + (os.getpid() % 1000)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, results)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(results)
    f0, t0, g0 = res[0]
    f1, t1, _ = res[1]
    assert t0 == t1 == 2.0                       # max over ranks
    assert not set(f0) & set(f1)                 # disjoint frames
    assert sorted(f0 + f1) == [(10 + i) % 120 for i in range(24)]
    assert g0[1] == f1
    assert replicas.whole_job_rate(12, world, t0) == pytest.approx(12.0)


def test_single_process_identity():
    assert replicas.reduce_max(3.5) == 3.5
    assert replicas.frames_for_rank(0, 1, 0, 3, 120) == [0, 1, 2]
    with pytest.raises(ValueError):
        replicas.frame_index(2, 2, 0, 120)


def _dying_worker(rank, world, port, results):
    """Rank 1 leaves between steps, before the timing reduction; rank 0 must
    get an error from the reduction within the group's timeout, not hang."""
    import datetime
    import time

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(3)                       # no further collective from this rank
    t = time.monotonic()
    try:
        replicas.reduce_max(1.0, dist)
        results[rank] = ("returned", time.monotonic() - t)
    except Exception as e:               # gloo reports the lost peer or the timeout
        results[rank] = (type(e).__name__, time.monotonic() - t)
    os._exit(0)


def test_lost_rank_fails_the_reduction_instead_of_hanging():
    world = 2
    port = 30500 + (os.getpid() % 1000)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        procs = [ctx.Process(target=_dying_worker, args=(r, world, port, results)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert procs[1].exitcode == 3
        assert procs[0].exitcode == 0
        kind, seconds = dict(results)[0]
    assert kind != "returned"
    assert seconds < 60
