"""Parity of the CUDA path (libcgfd.so, through the C ABI) with the CPU
oracle on the same seeded inputs.

Tolerances: relative L2 <= 1e-4 for slip rate, slip, rupture time and
station velocity (the bar of the forward path); <= 2e-5 for whole
wavefields after a few steps from a random state.
"""
import dataclasses

import numpy as np
import pytest

import inputs
from cgfd import PEAK_FIELDS, Solver, WAVE_COMPONENTS
from oracle import OracleSolver

pytestmark = pytest.mark.gpu

TOL = 1e-4


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


def _pair(prob):
    return Solver(prob), OracleSolver(prob)


@pytest.mark.parametrize("method,free", [(2, 1), (1, 1), (2, 0)])
def test_random_state_steps(cgfd_lib, oracle_built, method, free):
    """Eight steps (all eight operator pairs) from a random wavefield: every
    volume, boundary and fault operator contributes."""
    p = inputs.small_planar(nt=10, dynamic_method=method, free_surface=free)
    rng = np.random.default_rng(11)
    g, o = _pair(p)
    for c in range(9):
        scale = 1e-3 if c < 3 else 1e3
        f = (rng.standard_normal((p.nk, p.nj, p.ni)) * scale).astype(np.float32)
        g.set_wavefield(c, f)
        o.set_wavefield(c, f)
    for step in range(8):
        g.run(1)
        o.run(1)
        for c in range(9):
            e = rel_l2(g.wavefield(c), o.wavefield(c))
            assert e < 2e-5, f"step {step} {WAVE_COMPONENTS[c]} rel-L2 {e:.2e}"


@pytest.mark.parametrize("method,free", [(2, 1), (1, 1), (2, 0)])
def test_rupture_small(cgfd_lib, oracle_built, method, free):
    nt = 80
    p = inputs.small_planar(nt=nt, dynamic_method=method, free_surface=free)
    g, o = _pair(p)
    vs_g, vs_o = [], []
    for _ in range(nt // 10):
        g.run(10)
        o.run(10)
        vs_g.append(g.fault("Vs"))
        vs_o.append(o.fault("Vs"))
    vs_g, vs_o = np.array(vs_g), np.array(vs_o)
    assert vs_o.max() > 0.1, "no rupture in the oracle run"
    assert rel_l2(vs_g, vs_o) < TOL
    for f in ("Slip", "Slip1", "Peak_vs", "Tn", "Ts1"):
        assert rel_l2(g.fault(f), o.fault(f)) < TOL, f
    t0g, t0o = g.fault("Init_t0"), o.fault("Init_t0")
    rup = t0o > 0
    assert rup.sum() > 20
    assert np.array_equal(t0g > 0, rup)
    assert rel_l2(t0g[rup], t0o[rup]) < TOL
    sg, so = g.stations(), o.stations()
    assert sg.shape == so.shape == (len(p.stations), 9, nt)
    assert rel_l2(sg[:, :3], so[:, :3]) < TOL
    fg, fo = g.fault_stations(), o.fault_stations()
    assert rel_l2(fg, fo) < TOL
    for c in range(9):
        assert rel_l2(g.wavefield(c), o.wavefield(c)) < TOL, WAVE_COMPONENTS[c]


def test_checkpoint_restore(cgfd_lib):
    p = inputs.small_planar(nt=40)
    g = Solver(p)
    g.run(13)
    buf = g.checkpoint()
    g.run(20)
    ref = g.fault("Slip").copy(), g.wavefield("Vy").copy(), g.surface_peaks()
    g.restore(buf)
    assert g.steps_done == 13
    g.run(20)
    assert np.array_equal(g.fault("Slip"), ref[0])
    assert np.array_equal(g.wavefield("Vy"), ref[1])
    assert np.array_equal(g.surface_peaks(), ref[2])


def test_graph_and_direct_launch_agree(cgfd_lib, monkeypatch):
    p = inputs.small_planar(nt=20)
    g1 = Solver(p)
    g1.run(17)
    monkeypatch.setenv("CGFD_NO_GRAPH", "1")
    g2 = Solver(p)
    g2.run(17)
    assert np.array_equal(g1.fault("Vs"), g2.fault("Vs"))
    assert np.array_equal(g1.wavefield("Txy"), g2.wavefield("Txy"))


def test_unstable_run_reports_error(cgfd_lib):
    p = inputs.small_planar(nt=400, dt=0.05)
    p.check_stability = 0
    g = Solver(p)
    with pytest.raises(Exception, match="ERR_UNSTABLE"):
        g.run(400)


def test_dt_above_limit_rejected(cgfd_lib):
    p = inputs.small_planar(nt=10, dt=0.05)
    with pytest.raises(Exception, match="ERR_DT"):
        Solver(p)


def _sponge(p, layers=6, vel=6000.0):
    """The same problem with an exponential sponge on the five non-surface
    faces in place of the CFS-PML."""
    top = 0 if p.free_surface else layers
    return dataclasses.replace(p, pml_layers=((0, 0), (0, 0), (0, 0)),
                               ablexp_layers=((layers, layers), (layers, layers), (layers, top)),
                               ablexp_ref_vel=((vel, vel), (vel, vel), (vel, vel)))


@pytest.mark.parametrize("free", [1, 0])
def test_sponge_random_state_steps(cgfd_lib, oracle_built, free):
    """Eight steps from a random wavefield with the sponge instead of the
    PML: the end-of-step masks, and with a free surface the surface peaks."""
    p = _sponge(inputs.small_planar(nt=10, pml=0, free_surface=free))
    rng = np.random.default_rng(12)
    g, o = _pair(p)
    for c in range(9):
        scale = 1e-3 if c < 3 else 1e3
        f = (rng.standard_normal((p.nk, p.nj, p.ni)) * scale).astype(np.float32)
        g.set_wavefield(c, f)
        o.set_wavefield(c, f)
    for step in range(8):
        g.run(1)
        o.run(1)
        for c in range(9):
            e = rel_l2(g.wavefield(c), o.wavefield(c))
            assert e < 2e-5, f"step {step} {WAVE_COMPONENTS[c]} rel-L2 {e:.2e}"
    if free:
        pg, po = g.surface_peaks(), o.surface_peaks()
        for c, name in enumerate(PEAK_FIELDS):
            assert rel_l2(pg[c], po[c]) < 2e-5, name


def test_rupture_sponge_and_peaks(cgfd_lib, oracle_built):
    """A rupture with the sponge boundary: fault outputs, stations and the
    free-surface peak velocity, acceleration and displacement."""
    nt = 80
    p = _sponge(inputs.small_planar(nt=nt, pml=0))
    g, o = _pair(p)
    g.run(nt)
    o.run(nt)
    assert o.fault("Vs").max() > 0.1, "no rupture in the oracle run"
    for f in ("Vs", "Slip", "Peak_vs", "Tn", "Ts1"):
        assert rel_l2(g.fault(f), o.fault(f)) < TOL, f
    assert rel_l2(g.stations()[:, :3], o.stations()[:, :3]) < TOL
    pg, po = g.surface_peaks(), o.surface_peaks()
    assert po[0].max() > 0
    for c, name in enumerate(PEAK_FIELDS):
        assert rel_l2(pg[c], po[c]) < TOL, name


def test_surface_peaks_with_pml(cgfd_lib, oracle_built):
    """Peaks of the PML case of the rupture tests (the configuration the
    benchmarks run)."""
    nt = 60
    p = inputs.small_planar(nt=nt)
    g, o = _pair(p)
    g.run(nt)
    o.run(nt)
    pg, po = g.surface_peaks(), o.surface_peaks()
    for c, name in enumerate(PEAK_FIELDS):
        assert rel_l2(pg[c], po[c]) < TOL, name


def test_no_surface_peaks_without_free_surface(cgfd_lib):
    g = Solver(inputs.small_planar(nt=10, free_surface=0))
    with pytest.raises(Exception, match="ERR_ARG"):
        g.surface_peaks()


def test_sponge_with_pml_rejected(cgfd_lib):
    p = dataclasses.replace(inputs.small_planar(nt=10), ablexp_layers=((4, 4), (0, 0), (0, 0)))
    with pytest.raises(Exception, match="ERR_ARG"):
        Solver(p)


def test_error_against_fp64(cgfd_lib, oracle_built):
    """Error of the float32 CUDA path against the FP64 build of the same
    scheme (the double-precision oracle), beside the error of the float32
    oracle, which does the reference's float arithmetic: the CUDA path may
    differ from FP64 only as much as float32 arithmetic of the scheme does."""
    nt = 80
    p = inputs.small_planar(nt=nt)
    g, o32, o64 = Solver(p), OracleSolver(p), OracleSolver(p, double=True)
    for s in (g, o32, o64):
        s.run(nt)
    errs = {}
    for f in ("Vs", "Slip", "Peak_vs", "Ts1"):
        ref = o64.fault(f)
        errs[f] = (rel_l2(g.fault(f), ref), rel_l2(o32.fault(f), ref))
    ref = o64.stations()[:, :3]
    errs["stations"] = (rel_l2(g.stations()[:, :3], ref), rel_l2(o32.stations()[:, :3], ref))
    print("rel-L2 vs FP64 (cuda, float oracle):", {k: (f"{a:.2e}", f"{b:.2e}") for k, (a, b) in errs.items()})
    for k, (gpu, f32) in errs.items():
        assert gpu < TOL, k
        assert gpu <= 4.0 * f32 + 1e-7, (k, gpu, f32)


def test_early_fault_kernels(cgfd_lib, oracle_built, monkeypatch):
    """A fault whose neighbourhood (i0 +- 6, split box + 3 nodes) stays clear of
    every PML slab and edge box: there a stage's first fault kernels start
    beside the previous stage's PML kernels.  The schedule changes no
    arithmetic, so the result equals the serial schedule's bit for bit, and
    the oracle's within the tolerance."""
    nt, L, margin = 60, 5, 10
    p = inputs.tpv_planar(ni=40, nj=80, nk=40, fault_x_index=21, fault_grid=[25, 56, 15, 40], nuc_half=3,
                          pml=L, nt=nt, nsta=4, margin=margin)
    i0 = p.fault_x_index[0] - 1
    # PML slabs and edges occupy the outer L + 1 nodes of x, y and the bottom
    assert i0 - 6 > L and i0 + 6 < p.ni - 1 - L
    assert margin - 3 > L and p.nj - 1 - margin + 3 < p.nj - 1 - L and margin - 3 > L
    g_early = Solver(p)
    monkeypatch.setenv("CGFD_PRE_EARLY", "0")
    g_serial = Solver(p)
    o = OracleSolver(p)
    for s in (g_early, g_serial, o):
        s.run(nt)
    assert o.fault("Vs").max() > 0.1
    for f in ("Vs", "Slip", "Tn", "Ts1"):
        assert np.array_equal(g_early.fault(f), g_serial.fault(f)), f
        assert rel_l2(g_early.fault(f), o.fault(f)) < TOL, f
    for c in range(9):
        assert np.array_equal(g_early.wavefield(c), g_serial.wavefield(c)), WAVE_COMPONENTS[c]


def test_interior_chunk_choice_changes_nothing(cgfd_lib, monkeypatch):
    """The autotuned y chunk of the interior kernel and a fixed small one give
    the same result bit for bit (the chunk only orders the blocks)."""
    p = inputs.small_planar(nt=12)
    g1 = Solver(p)
    monkeypatch.setenv("CGFD_INTERIOR_YCHUNK", "1")
    g2 = Solver(p)
    g1.run(12)
    g2.run(12)
    assert np.array_equal(g1.fault("Vs"), g2.fault("Vs"))
    for c in range(9):
        assert np.array_equal(g1.wavefield(c), g2.wavefield(c)), WAVE_COMPONENTS[c]


def test_interior_whole_tiles(cgfd_lib, monkeypatch):
    """The interior box is cut to a whole number of 32-point tiles in x and
    the columns left over join the right x PML slab, whose kernel adds the
    PML terms only inside the PML layers; with the cut switched off
    (CGFD_ALIGN_TILES=0) the last tile of each row runs them.  The x
    direction's sums are formed in the slab kernel's order there, so the two
    agree to rounding, not bit for bit.  48 points in x with a 5-layer PML:
    an interior box 36 wide, so 32 + 4 columns, the fault's neighbourhood in
    the first 32."""
    p = inputs.tpv_planar(ni=48, nj=80, nk=40, fault_x_index=15, fault_grid=[25, 56, 15, 40], nuc_half=3,
                          pml=5, nt=20, nsta=4, margin=10)
    g1 = Solver(p)
    monkeypatch.setenv("CGFD_ALIGN_TILES", "0")
    g2 = Solver(p)
    monkeypatch.delenv("CGFD_ALIGN_TILES")
    g1.run(17)
    g2.run(17)
    assert g1.last_launches() == g2.last_launches()
    _, _, pts1 = g1.kernel_timing(1)
    _, _, pts2 = g2.kernel_timing(1)
    assert pts2 - pts1 == 4 * (80 - 12) * (40 - 6 - 4), (pts1, pts2)
    for f in ("Vs", "Slip", "Tn", "Ts1"):
        assert rel_l2(g1.fault(f), g2.fault(f)) <= 1e-6, f
    for c in range(9):
        assert rel_l2(g1.wavefield(c), g2.wavefield(c)) <= 1e-6, WAVE_COMPONENTS[c]
    assert rel_l2(g1.stations(), g2.stations()) <= 1e-6


def test_pool_reuse_and_release(cgfd_lib):
    """Solver memory comes from the device's memory pool: a solver made after
    another was destroyed reuses its blocks and runs the same, and the
    cached blocks can be handed back."""
    p = inputs.small_planar(nt=6)
    g = Solver(p)
    g.run(6)
    ref = g.wavefield("Vz").copy()
    g.close()
    g2 = Solver(p)
    g2.run(6)
    assert np.array_equal(g2.wavefield("Vz"), ref)
    g2.close()
    assert cgfd_lib.cgfd_release_cached_memory() == 0


@pytest.mark.parametrize("env", [("CGFD_BRANCHES", "0"), ("CGFD_BRANCHES", "1"), ("CGFD_BRANCHES", "2"),
                                 ("CGFD_PRE_OVERLAP", "0"), ("CGFD_POST_EARLY", "0")])
def test_stage_schedules_agree(cgfd_lib, monkeypatch, env):
    """Every stage schedule (one stream; fault, interior and PML kernels side
    by side; the interior kernel alone, then the fault slabs beside the PML
    kernels; the default, with the y / z PML slabs on a third stream, the
    stage's first fault kernels beside the interior kernel and the fault
    planes after them, and the fault slabs right after the first fault
    kernels; each of those last two switched off) changes no arithmetic: the
    same result bit for bit, on a case whose fault neighbourhood stays clear
    of the PML boxes (so the next stage's fault kernels also start early)
    and one whose fault reaches them."""
    key, val = env
    cases = [inputs.tpv_planar(ni=40, nj=80, nk=40, fault_x_index=21, fault_grid=[25, 56, 15, 40], nuc_half=3,
                               pml=5, nt=20, nsta=4, margin=10),
             inputs.small_planar(nt=20)]
    for p in cases:
        ref = Solver(p)
        ref.run(17)
        monkeypatch.setenv(key, val)
        g = Solver(p)
        monkeypatch.delenv(key)
        g.run(17)
        for f in ("Vs", "Slip", "Tn", "Ts1"):
            assert np.array_equal(ref.fault(f), g.fault(f)), (p.name, f)
        for c in range(9):
            assert np.array_equal(ref.wavefield(c), g.wavefield(c)), (p.name, WAVE_COMPONENTS[c])
        assert np.array_equal(ref.stations(), g.stations()), p.name


def test_surface_rows_kernels_agree(cgfd_lib, monkeypatch):
    """The rows under the free surface away from the PML columns run in a
    kernel of their own, the shell's code without the PML faces; with it
    switched off (CGFD_TOP=0) the shell kernel updates all surface rows.
    Without the PML terms the compiler fuses some multiply-adds of the
    direction sums differently, so the two agree to rounding (relative L2
    <= 1e-6 after 17 steps, measured ~3e-8), not bit for bit."""
    cases = [inputs.tpv_planar(ni=40, nj=80, nk=40, fault_x_index=21, fault_grid=[25, 56, 15, 40], nuc_half=3,
                               pml=5, nt=20, nsta=4, margin=10),
             inputs.small_planar(nt=20, dynamic_method=2)]
    for p in cases:
        ref = Solver(p)
        ref.run(17)
        monkeypatch.setenv("CGFD_TOP", "0")
        g = Solver(p)
        monkeypatch.delenv("CGFD_TOP")
        g.run(17)
        if p is cases[0]:
            # PML columns on every side: one launch more per stage with the
            # surface rows split
            assert ref.last_launches() == g.last_launches() + 4 * 17, (ref.last_launches(), g.last_launches())
        for f in ("Vs", "Slip", "Tn", "Ts1"):
            assert rel_l2(ref.fault(f), g.fault(f)) <= 1e-6, (p.name, f)
        for c in range(9):
            assert rel_l2(ref.wavefield(c), g.wavefield(c)) <= 1e-6, (p.name, WAVE_COMPONENTS[c])
        assert rel_l2(ref.stations(), g.stations()) <= 1e-6, p.name
