"""Replica timing across ranks (bench.py --gpus N), on CPU with gloo.

Each rank reports its own run time; every rank must see the slowest one,
and the aggregate rate is the points of all replicas over that time."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, times, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(ws),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    import replicas
    w, r, _ = replicas.init("gloo", timeout_s=60)
    assert (w, r) == (ws, rank)
    replicas.barrier(w)
    m = replicas.allmax(w, times[rank], device="cpu")
    rate = replicas.aggregate_rate(1000, 10, w, m)
    replicas.barrier(w)
    replicas.finish(w)
    out.put((rank, m, rate))


@pytest.mark.parametrize("ws", [2, 3])
def test_replica_max_over_ranks(ws):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    times = [0.5 + 0.25 * r for r in range(ws)]
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, times, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, rate in res:
        assert m == max(times)
        assert rate == pytest.approx(1000 * 10 * ws / max(times))


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    import replicas
    assert replicas.init("gloo") == (1, 0, 0)
    assert replicas.allmax(1, 3.5, device="cpu") == 3.5
    assert replicas.aggregate_rate(10, 2, 1, 4.0) == 5.0
