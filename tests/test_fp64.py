"""The double build of the solver's kernels (libcgfd64.so).

The same CUDA sources built with -DCGFD_FP64 compute and store every value
in double behind the same C ABI.  CPU: the library loads and exports every
entry point include/cgfd.h declares.  GPU: the double build agrees with the
double-precision oracle to rounding level (it is the same scheme), and the
float build's error is stated against it on the 160x100x80 planar case
(600 steps), beside the error of the float oracle, which does the
reference's float arithmetic."""
import json
import os

import numpy as np
import pytest

import inputs
from conftest import ROOT

FIELDS = ("Vs", "Slip", "Peak_vs", "Tn", "Ts1")


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def lib64(cgfd_lib):
    import cgfd
    return cgfd.load_library64()


def test_fp64_library_exports_all(lib64):
    from test_abi import declared_functions
    missing = [n for n in declared_functions() if not hasattr(lib64, n)]
    assert not missing, missing
    assert lib64.cgfd_abi_version() == 2


@pytest.mark.gpu
def test_fp64_build_matches_fp64_oracle(lib64, oracle_built):
    """The double build against the double oracle on the small split-node
    case: agreement at the level of double rounding carried through 60
    steps of a rupture (far below anything float arithmetic reaches)."""
    from cgfd import Solver
    from oracle import OracleSolver
    p = inputs.small_planar(nt=60)
    g, o = Solver(p, lib=lib64), OracleSolver(p, double=True)
    g.run(60)
    o.run(60)
    assert o.fault("Vs").max() > 0.1
    for f in FIELDS:
        # the outputs are narrowed to float on read-back: half an ulp of float
        assert rel_l2(g.fault(f), o.fault(f)) < 1e-6, f
    assert rel_l2(g.stations()[:, :3], o.stations()[:, :3]) < 1e-6


@pytest.mark.gpu
def test_float_error_against_fp64_kernels(cgfd_lib, lib64, oracle_built, tmp_path):
    """Relative L2 error of the float CUDA path against the double build of
    the same kernels on the 160x100x80 planar case, 600 steps: below 1e-4 on
    slip rate, slip, peak slip rate, tractions and station velocity, and of
    the size of the float oracle's own error (the reference's float
    arithmetic) against the same double solution."""
    from cgfd import Solver
    from oracle import OracleSolver
    nt = 600
    p = inputs.tpv_planar()
    g32, g64, o32 = Solver(p), Solver(p, lib=lib64), OracleSolver(p)
    for s in (g32, g64, o32):
        s.run(nt)
    errs = {}
    for f in FIELDS:
        ref = g64.fault(f)
        errs[f] = (rel_l2(g32.fault(f), ref), rel_l2(o32.fault(f), ref))
    ref = g64.stations()[:, :3]
    errs["station velocity"] = (rel_l2(g32.stations()[:, :3], ref), rel_l2(o32.stations()[:, :3], ref))
    t64, t32 = g64.fault("Init_t0"), g32.fault("Init_t0")
    rup = t64 > 0
    assert np.array_equal(t32 > 0, rup)
    errs["rupture time (max |dt|/dt)"] = (float(np.abs(t32[rup] - t64[rup]).max() / p.dt), None)
    print("rel-L2 vs the FP64 kernels (float CUDA, float oracle):",
          {k: (f"{a:.2e}", None if b is None else f"{b:.2e}") for k, (a, b) in errs.items()})
    out = os.environ.get("CGFD_FP64_REPORT")
    if out:
        with open(out, "w") as fh:
            json.dump({"case": p.name, "steps": nt, "rel_l2_vs_fp64_kernels": errs}, fh, indent=1)
    for k, (cu, f32) in errs.items():
        if f32 is None:
            assert cu <= 1.0 + 1e-4, k          # rupture front within one time step
            continue
        assert cu < 1e-4, (k, cu)
        assert cu <= 4.0 * f32 + 1e-7, (k, cu, f32)
