"""Ensembles of rupture scenarios sharded across GPUs, one process per GPU.

Scenarios are independent units: there is no exchange step between them.
Each rank takes a share of the scenarios chosen by cost, runs its share as
one ensemble on its own GPU (cgfd_ensemble_*), and the per-scenario outputs
are gathered on rank 0 in scenario order.  The only collectives are the
final gather and the timing reduction; nothing crosses GPUs while the
scenarios step.  The reference runs one scenario per MPI job
(src/forward/main_curv_col_el_3d.cu:26-65) and has no counterpart.

Cost of a scenario: grid points x steps (the forward step is HBM-bound at a
fixed number of bytes per point and step).  ``partition`` is the
longest-processing-time-first rule: scenarios in decreasing cost, each to
the rank with the least cost so far (ties to the lower rank), which keeps
the slowest rank within 4/3 of the optimum.
"""
from __future__ import annotations

from typing import Callable, Sequence


def scenario_cost(prob, nsteps: int) -> int:
    return int(prob.points) * int(nsteps)


def partition(costs: Sequence[float], nranks: int) -> list[list[int]]:
    """Scenario indices per rank, each list in increasing index order."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    load = [0.0] * nranks
    parts: list[list[int]] = [[] for _ in range(nranks)]
    for q in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(nranks), key=lambda x: (load[x], x))
        parts[r].append(q)
        load[r] += costs[q]
    return [sorted(p) for p in parts]


def gather_on_root(ws: int, rank: int, items: dict) -> dict | None:
    """Merge every rank's {scenario index: result} on rank 0 (None on the
    other ranks).  Results travel as pickled host objects over the process
    group (gloo, or NCCL with the current device set)."""
    if ws <= 1:
        return dict(items)
    import torch.distributed as dist
    out = [None] * ws if rank == 0 else None
    dist.gather_object(items, out, dst=0)
    if rank != 0:
        return None
    merged: dict = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"scenario {k} returned by two ranks")
            merged[k] = v
    return merged


def run_sharded(probs: Sequence, nsteps: int, ws: int, rank: int,
                runner: Callable[[list, int], list]) -> list | None:
    """Run every scenario for nsteps, sharded over ws ranks; on rank 0 the
    list of results in scenario order, None elsewhere.  ``runner(problems,
    nsteps)`` advances this rank's problems and returns one result each."""
    parts = partition([scenario_cost(p, nsteps) for p in probs], ws)
    mine = parts[rank]
    res = runner([probs[q] for q in mine], nsteps) if mine else []
    if len(res) != len(mine):
        raise RuntimeError("runner returned a wrong number of results")
    merged = gather_on_root(ws, rank, dict(zip(mine, res)))
    if merged is None:
        return None
    missing = [q for q in range(len(probs)) if q not in merged]
    if missing:
        raise RuntimeError(f"scenarios without a result: {missing}")
    return [merged[q] for q in range(len(probs))]


FAULT_OUTPUTS = ("Vs", "Slip", "Peak_vs", "Init_t0", "Tn", "Ts1")


def ensemble_runner(probs: list, nsteps: int) -> list:
    """GPU runner: the rank's scenarios as one ensemble on the current
    device; per scenario the fault output fields and the station traces as
    host arrays."""
    import cgfd
    solvers = [cgfd.Solver(p) for p in probs]
    ens = cgfd.Ensemble(solvers)
    ens.run(nsteps)
    out = []
    for p, s in zip(probs, solvers):
        r = {f: s.fault(f) for f in FAULT_OUTPUTS}
        r["stations"] = s.stations()
        r["name"] = p.name
        out.append(r)
    ens.close()
    for s in solvers:
        s.close()
    return out
