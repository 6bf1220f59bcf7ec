"""The replica plumbing of bench.py on CPU: two gloo ranks (processes) that
each time their own work agree on the slowest rank's time, and the whole-job
rate counts every rank's work over it."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from codens_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=60)
    try:
        rep.barrier()
        seconds = 0.010 * (rank + 1)          # rank 1 is the slow one
        out[rank] = (rep.max(seconds), rep.rate(1000.0, seconds))
        rep.barrier()
    finally:
        rep.close()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(90)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        for r in range(2):
            slowest, rate = out[r]
            assert slowest == pytest.approx(0.020)
            assert rate == pytest.approx(2 * 1000.0 / 0.020)


def test_single_process_needs_no_process_group(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    from codens_b200.replicas import Replicas
    rep = Replicas("gloo")
    assert rep.world == 1
    assert rep.max(0.5) == 0.5
    assert rep.rate(10.0, 2.0) == 5.0
    rep.close()
