"""The CUDA path against the golden fixtures and the scheme's known answers,
and its parity with the oracle on a curvilinear layered grid and on a box
without a fault.  All calls go through the C ABI (libcgfd.so)."""
import os

import numpy as np
import pytest

import cases
import inputs
from cgfd import Solver, WAVE_COMPONENTS
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(np.asarray(b, np.float64)), 1e-30))


@pytest.mark.parametrize("method", [1, 2])
def test_golden_fixture(cgfd_lib, method):
    """30 steps of the 36x56x32 split-node case against the double-precision
    oracle's fixture: relative L2 <= 2e-4 on every field."""
    import make_golden
    g = np.load(os.path.join(GOLDEN, f"small_planar_m{method}_{make_golden.NSTEPS}.npz"))
    p = inputs.small_planar(dynamic_method=method, nt=make_golden.NSTEPS)
    s = Solver(p)
    s.run(make_golden.NSTEPS)
    snap = make_golden.snapshot(s, p)
    for k in g.files:
        assert snap[k].shape == g[k].shape, k
        assert rel_l2(snap[k], g[k]) < 2e-4, (k, rel_l2(snap[k], g[k]))


def test_linear_velocity_one_step(cgfd_lib):
    from test_oracle import _linear_fields, check_linear_step
    p = cases.uniform_box(ni=40, nj=40, nk=40, nt=2)
    V, G = _linear_fields(p)
    s = Solver(p)
    for c, v in V.items():
        s.set_wavefield(c, v)
    s.run(1)
    check_linear_step(s, p, V, G)


def test_fault_below_strength_stays_locked(cgfd_lib):
    p = inputs.small_planar(nt=20)
    p.T0y[0][:] = 60.0e6
    s = Solver(p)
    s.run(20)
    assert s.fault("Vs").max() <= 1e-12
    assert s.fault("Slip").max() == 0.0
    for c in range(9):
        assert np.abs(s.wavefield(c)).max() == 0.0, WAVE_COMPONENTS[c]


def test_no_fault_pulse_with_pml_and_free_surface(cgfd_lib, oracle_built):
    """No fault: a pulse in a box with CFS-PML on five faces and a free
    surface, 24 steps (three cycles of the operator pairs)."""
    from oracle import OracleSolver
    p = cases.uniform_box(ni=40, nj=44, nk=36, pml=6, free_surface=1, nt=30)
    gs = cases.gaussian(p, (20, 22, 30), 400.0)
    s, o = Solver(p), OracleSolver(p)
    for solver in (s, o):
        solver.set_wavefield("Vx", gs)
        solver.set_wavefield("Vz", -0.7 * gs)
        solver.set_wavefield("Txy", 1e6 * gs)
        solver.run(24)
    for c in range(9):
        assert rel_l2(s.wavefield(c), o.wavefield(c)) < 1e-4, WAVE_COMPONENTS[c]


@pytest.mark.parametrize("method", [1, 2])
def test_hills_layered_small(cgfd_lib, oracle_built, method):
    """Curvilinear grid under Gaussian hills, layered perturbed medium,
    stations on the topography: the benchmark workload's construction at
    48x72x40, 60 steps."""
    from oracle import OracleSolver
    nt = 60
    p = inputs.hills_layered(ni=48, nj=72, nk=40, h=100.0, pml=8, nsta=6, fault_len=48, fault_depth=30,
                             margin=6, dynamic_method=method, nt=nt, nhills=3)
    s, o = Solver(p), OracleSolver(p)
    s.run(nt)
    o.run(nt)
    assert o.fault("Vs").max() > 0.1, "no rupture in the oracle run"
    for f in ("Vs", "Slip", "Peak_vs", "Tn", "Ts1"):
        assert rel_l2(s.fault(f), o.fault(f)) < 1e-4, f
    t0s, t0o = s.fault("Init_t0"), o.fault("Init_t0")
    assert np.array_equal(t0s > 0, t0o > 0)
    assert rel_l2(s.stations()[:, :3], o.stations()[:, :3]) < 1e-4
    for c in range(9):
        assert rel_l2(s.wavefield(c), o.wavefield(c)) < 1e-4, WAVE_COMPONENTS[c]


def test_tpv_planar_full_600_steps(cgfd_lib, oracle_built):
    """The 160x100x80 planar case in full (h = 200 m, 10-layer PML, flat
    free surface, 600 steps of 0.01 s): slip rate, slip, peak slip rate and
    station velocity within relative L2 1e-4 of the oracle, the rupture time
    of every node within one time step, the same set of ruptured nodes."""
    from oracle import OracleSolver
    p = inputs.tpv_planar()
    s, o = Solver(p), OracleSolver(p)
    s.run(600)
    o.run(600)
    for f in ("Vs", "Slip", "Peak_vs", "Tn", "Ts1"):
        assert rel_l2(s.fault(f), o.fault(f)) < 1e-4, f
    t0s, t0o = s.fault("Init_t0"), o.fault("Init_t0")
    rup = t0o > 0
    assert rup.sum() > 1000
    assert np.array_equal(t0s > 0, rup)
    assert np.abs(t0s[rup] - t0o[rup]).max() <= p.dt * 1.0001
    assert rel_l2(s.stations()[:, :3], o.stations()[:, :3]) < 1e-4
    assert rel_l2(s.fault_stations(), o.fault_stations()) < 1e-4


@pytest.mark.parametrize("method", [1, 2])
def test_two_faults(cgfd_lib, oracle_built, method):
    """Two parallel faults, each with its own fault_grid, stress and friction:
    both ruptures, the fault stations of each and the wavefield between them."""
    from oracle import OracleSolver
    p = inputs.two_faults(dynamic_method=method, nt=60)
    s, o = Solver(p), OracleSolver(p)
    s.run(60)
    o.run(60)
    for f in range(2):
        assert o.fault("Vs", f).max() > 0.5
        for name in ("Vs", "Slip", "Peak_vs", "Tn", "Ts1"):
            assert rel_l2(s.fault(name, f), o.fault(name, f)) < 1e-4, (f, name)
        assert np.array_equal(s.fault("Init_t0", f) > 0, o.fault("Init_t0", f) > 0)
    assert rel_l2(s.fault_stations(), o.fault_stations()) < 1e-4
    assert rel_l2(s.stations()[:, :3], o.stations()[:, :3]) < 1e-4
    for c in range(9):
        assert rel_l2(s.wavefield(c), o.wavefield(c)) < 1e-4, WAVE_COMPONENTS[c]


def test_dipping_fault_small(cgfd_lib, oracle_built):
    """A 25-degree dipping fault meshed into a sheared curvilinear grid under
    hills, von Karman shear stress: 40 steps against the oracle."""
    from oracle import OracleSolver
    p = inputs.hills_layered(ni=64, nj=96, nk=48, h=50.0, pml=8, nsta=4, fault_len=64, fault_depth=36, margin=6,
                             nt=40, nhills=3, dip=25.0, vk_stress=True, nuc_half=6)
    s, o = Solver(p), OracleSolver(p)
    s.run(40)
    o.run(40)
    assert o.fault("Vs").max() > 0.5
    for f in ("Vs", "Slip", "Peak_vs", "Tn", "Ts1", "Ts2"):
        assert rel_l2(s.fault(f), o.fault(f)) < 1e-4, f
    assert rel_l2(s.stations()[:, :3], o.stations()[:, :3]) < 1e-4
    for c in range(9):
        assert rel_l2(s.wavefield(c), o.wavefield(c)) < 1e-4, WAVE_COMPONENTS[c]
