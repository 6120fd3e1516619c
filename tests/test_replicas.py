"""Multi-GPU plumbing of bench.py and the sweeps, on CPU with the gloo
backend and two processes: barrier, max / sum over ranks, and the sharding of
sweep members (each member on exactly one rank)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from gpesolver_b200 import replicas, sweep

    w, r, _ = replicas.env()
    replicas.init(w, r, "gloo", timeout_s=60)
    replicas.barrier(w)
    mx = replicas.reduce(w, float(10 + r), "max", "gloo")
    sm = replicas.reduce(w, float(10 + r), "sum", "gloo")
    members = sweep.sweep_json(count=7, seed=0)
    mine = replicas.shard(list(range(len(members))), r, w)
    total = replicas.reduce(w, float(len(mine)), "sum", "gloo")
    replicas.finish(w)
    out[rank] = (mx, sm, tuple(mine), total)


def test_two_rank_gloo_reductions_and_sharding():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, out)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 11.0
    assert out[0][1] == out[1][1] == 21.0
    assert sorted(out[0][2] + out[1][2]) == list(range(7))
    assert out[0][3] == out[1][3] == 7.0
