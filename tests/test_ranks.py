"""The N > 1 bookkeeping of bench.py (replicas): two gloo ranks on the CPU
agree on the slowest rank's time and on the whole-job rate, and take the same
collectives in the same order."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, results):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank),
                       "LOCAL_RANK": str(rank), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    from spmv_b200 import ranks
    info = ranks.init("gloo", timeout_s=60)
    ranks.barrier(info)
    # Rank r "took" 1 + r seconds for 10 solves.
    rate = ranks.whole_job_rate(10, 1.0 + rank, info)
    tmax = ranks.max_over_ranks(1.0 + rank, info)
    ranks.barrier(info)
    results[rank] = (rate, tmax)
    ranks.finalize(info)


def test_two_gloo_ranks_agree():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    results = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert results[0] == results[1]
    rate, tmax = results[0]
    assert tmax == 2.0 and rate == pytest.approx(2 * 10 / 2.0)


def test_single_rank_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from spmv_b200 import ranks
    info = ranks.init("gloo")
    assert (info.world, info.rank) == (1, 0)
    assert ranks.whole_job_rate(5, 2.0, info) == 2.5
