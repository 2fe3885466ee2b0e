"""Generate the golden fixtures in this folder from the double-precision
CPU oracle.

    python tests/golden/make_golden.py

Writes ``small_planar_m{1,2}_30.npz``: the 36x56x32 split-node case
(``inputs.small_planar``, dynamic_method 1 and 2) after 30 steps -- the 11
fault output fields, the station and fault-station traces, and two planes of
Vx, Vy, Txy (the plane i = i0 + 1 next to the fault and the plane j = 27
across it).  The float32 oracle and the CUDA path are both checked against
these arrays.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
sys.path[:0] = [os.path.join(ROOT, "gpu-cgfd3d-dynamic_b200"), os.path.join(ROOT, "oracle")]

import inputs  # noqa: E402
from cgfd import FAULT_FIELDS  # noqa: E402
from oracle import OracleSolver  # noqa: E402

NSTEPS = 30
PLANE_J = 27


def snapshot(solver, prob):
    i0 = prob.fault_x_index[0] - 1
    out = {f"fault_{f}": solver.fault(f) for f in FAULT_FIELDS}
    out["stations"] = solver.stations()
    out["fault_stations"] = solver.fault_stations()
    for c in ("Vx", "Vy", "Txy"):
        w = solver.wavefield(c)
        out[f"{c}_i0p1"] = w[:, :, i0 + 1]
        out[f"{c}_j{PLANE_J}"] = w[:, PLANE_J, :]
    return out


def main():
    for m in (1, 2):
        p = inputs.small_planar(dynamic_method=m, nt=NSTEPS)
        o = OracleSolver(p, double=True)
        o.run(NSTEPS)
        snap = {k: np.asarray(v, np.float32) for k, v in snapshot(o, p).items()}
        path = os.path.join(HERE, f"small_planar_m{m}_{NSTEPS}.npz")
        np.savez_compressed(path, **snap)
        print(path, sum(v.nbytes for v in snap.values()), "bytes")


if __name__ == "__main__":
    main()
