"""Ensemble scenarios sharded across ranks (shard.py), on CPU with gloo.

The partition is checked for balance and completeness; a world-size-2 run
uses the CPU oracle as each rank's runner (the GPU runner advances the
rank's share as one ensemble on its own device, which needs a GPU per rank)
and the gathered results must equal each scenario run on its own.
Unmeasured on GPU hardware: the pool gives one GPU per call."""
import os
import socket

import numpy as np
import pytest

import shard


def test_partition_is_complete_and_balanced():
    rng = np.random.default_rng(3)
    costs = list(rng.integers(1, 1000, 64))
    for n in (1, 2, 3, 8):
        parts = shard.partition(costs, n)
        assert sorted(q for p in parts for q in p) == list(range(64))
        loads = [sum(costs[q] for q in p) for p in parts]
        # longest-processing-time-first: the heaviest rank is within the
        # largest single cost of the mean
        assert max(loads) <= sum(costs) / n + max(costs)
    assert shard.partition([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    assert shard.partition([1, 9, 1, 1], 2) == [[1], [0, 2, 3]]
    with pytest.raises(ValueError):
        shard.partition([1], 0)


def test_partition_with_more_ranks_than_scenarios():
    parts = shard.partition([3, 1], 4)
    assert parts == [[0], [1], [], []]


def _problems():
    import inputs
    return [inputs.small_planar(nt=4, seed=s, dynamic_method=m) for s, m in ((7, 2), (8, 1), (9, 2))]


def _oracle_runner(probs, nsteps):
    from oracle import OracleSolver
    out = []
    for p in probs:
        o = OracleSolver(p, threads=2)
        o.run(nsteps)
        out.append({"Vs": o.fault("Vs"), "Slip": o.fault("Slip"), "stations": o.stations()})
        o.close()
    return out


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, nsteps, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(ws),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    import replicas
    w, r, _ = replicas.init("gloo", timeout_s=120)
    res = shard.run_sharded(_problems(), nsteps, w, r, _oracle_runner)
    replicas.barrier(w)
    replicas.finish(w)
    q.put((rank, res))


def test_sharded_run_gathers_every_scenario(oracle_built):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ws, nsteps, port = 2, 3, _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, nsteps, q)) for r in range(ws)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[1] is None
    res = got[0]
    want = _oracle_runner(_problems(), nsteps)
    assert len(res) == len(want)
    for a, b in zip(res, want):
        for k in b:
            assert np.array_equal(a[k], b[k]), k
    # the shares were split between the ranks
    parts = shard.partition([shard.scenario_cost(p, nsteps) for p in _problems()], ws)
    assert all(parts)
