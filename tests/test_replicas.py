"""Multi-rank path of the benchmark (replicas) on CPU with gloo, world size 2.

Each rank reports its own units and device time; the job throughput is the sum
of units over the slowest rank's time.  A missing rank must end the collective
with an error, not hang.
"""
import importlib
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q, mode):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    R = importlib.import_module("dennou-ogcm_b200.replicas")
    try:
        if mode == "missing" and rank == 1:
            return  # this rank never joins
        rep = R.Replicas("gloo", timeout_s=5 if mode == "missing" else 60)
        rep.barrier()
        units = 100.0 * (rank + 1)      # 100 and 200 field-levels
        secs = 0.5 if rank == 0 else 2.0
        out = {"max": rep.max(secs), "sum": rep.sum(units), "tp": rep.throughput(units, secs)}
        rep.barrier()
        rep.close()
        q.put((rank, "ok", out))
    except Exception as ex:  # the missing-rank case lands here
        q.put((rank, "error", type(ex).__name__))


def _run(mode, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, mode)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    res = []
    while not q.empty():
        res.append(q.get())
    for p in procs:
        if p.is_alive():
            p.kill()
    return res


def test_replica_reductions_gloo_world2():
    res = _run("ok")
    assert len(res) == 2
    for rank, status, out in res:
        assert status == "ok", out
        assert out["max"] == 2.0
        assert out["sum"] == 300.0
        assert out["tp"] == pytest.approx(150.0)


def test_missing_rank_fails_instead_of_hanging():
    res = _run("missing")
    # rank 1 never joins; rank 0 must come back with an error within the group timeout
    assert any(r == 0 and s == "error" for r, s, _ in res), res


def test_single_process_needs_no_group():
    R = importlib.import_module("dennou-ogcm_b200.replicas")
    rep = R.Replicas("gloo")
    assert not rep.active
    assert rep.max(3.0) == 3.0 and rep.sum(4.0) == 4.0
    assert rep.throughput(10.0, 2.0) == 5.0
