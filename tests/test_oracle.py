"""CPU tests of the oracle: known answers of the scheme and the golden fixtures.

The reference ships no tests, fixtures or CPU code for this path, so these
known-answer tests (exact metric of a uniform grid, exact Hooke update of a
linear velocity field, the CFL bound of a uniform grid, a fault below its
strength that never moves, a locked fault that converges to the welded
solution) are what pin the oracle's arithmetic.  The golden fixtures come
from the double-precision oracle (tests/golden/make_golden.py); the float32
oracle must reproduce them to rounding.
"""
import math
import os

import numpy as np
import pytest

import cases
import inputs

from conftest import GOLDEN


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(np.asarray(b, np.float64)), 1e-30))


@pytest.mark.parametrize("method", [1, 2])
def test_golden_float_oracle(oracle_built, method):
    """float32 oracle vs the double-precision fixture (30 steps, 36x56x32)."""
    import make_golden
    from oracle import OracleSolver
    g = np.load(os.path.join(GOLDEN, f"small_planar_m{method}_{make_golden.NSTEPS}.npz"))
    p = inputs.small_planar(dynamic_method=method, nt=make_golden.NSTEPS)
    o = OracleSolver(p)
    o.run(make_golden.NSTEPS)
    snap = make_golden.snapshot(o, p)
    assert set(snap) == set(g.files)
    for k in g.files:
        assert snap[k].shape == g[k].shape, k
        assert _rel(snap[k], g[k]) < 1e-4, (k, _rel(snap[k], g[k]))
    # the run ruptured: slip, a rupture front and peak slip rate above 1 m/s
    assert g["fault_Slip"].max() > 0.05
    assert g["fault_Peak_vs"].max() > 1.0
    assert (g["fault_Init_t0"] > 0).sum() > 100


def test_uniform_grid_metric(oracle_built):
    """Planar fault extrusion at h = 200 m: jac = h^3, xi_x = eta_y = zeta_z = 1/h."""
    from oracle import OracleSolver
    p = inputs.small_planar()
    o = OracleSolver(p)
    h = 200.0
    want = {0: h ** 3, 1: 1 / h, 5: 1 / h, 9: 1 / h}
    for cmp in range(10):
        m = o.metric(cmp)
        if cmp in want:
            np.testing.assert_allclose(m, want[cmp], rtol=1e-5)
        else:
            assert np.abs(m).max() < 1e-9, cmp


def test_uniform_grid_dt_max(oracle_built):
    """CFL bound of a uniform grid: 1.3 h / (sqrt(3) Vp) (the point-to-plane
    distance of calc_dtmax is h / sqrt(3))."""
    from oracle import OracleSolver
    p = cases.uniform_box(ni=16, nj=16, nk=16)
    o = OracleSolver(p)
    vp = math.sqrt((float(p.lam[0, 0, 0]) + 2 * float(p.mu[0, 0, 0])) / float(p.rho[0, 0, 0]))
    assert o.dt_max() == pytest.approx(1.3 * 100.0 / (math.sqrt(3.0) * vp), rel=1e-5)


def _linear_fields(p, h=100.0):
    k, j, i = np.meshgrid(np.arange(p.nk), np.arange(p.nj), np.arange(p.ni), indexing="ij")
    x, y, z = (i - p.ni // 2) * h, (j - p.nj // 2) * h, (k - p.nk + 1) * h
    G = np.array([[1e-3, 0.0, 2e-3], [1e-3, -5e-4, 0.0], [0.0, -3e-4, 7e-4]])   # G[c][b] = dV_c/dx_b
    V = {"Vx": G[0, 0] * x + G[0, 2] * z, "Vy": G[1, 0] * x + G[1, 1] * y, "Vz": G[2, 1] * y + G[2, 2] * z}
    return {c: v.astype(np.float32) for c, v in V.items()}, G


def hooke_after_one_step(p, G):
    lam, mu = float(p.lam[0, 0, 0]), float(p.mu[0, 0, 0])
    tr = G[0, 0] + G[1, 1] + G[2, 2]
    T = {"Txx": lam * tr + 2 * mu * G[0, 0], "Tyy": lam * tr + 2 * mu * G[1, 1], "Tzz": lam * tr + 2 * mu * G[2, 2],
         "Tyz": mu * (G[1, 2] + G[2, 1]), "Txz": mu * (G[0, 2] + G[2, 0]), "Txy": mu * (G[0, 1] + G[1, 0])}
    return {c: v * p.dt for c, v in T.items()}


def check_linear_step(solver, p, V, G):
    """Away from the boundaries (12 points per step for the 4 stages' 3-point
    reach), a linear velocity field is a steady state of the momentum
    equation and one RK4 step sets sigma = dt C grad V exactly: the DRP
    operators differentiate linear functions exactly."""
    sl = (slice(14, p.nk - 14), slice(14, p.nj - 14), slice(14, p.ni - 14))
    want = hooke_after_one_step(p, G)
    scale = max(abs(v) for v in want.values())
    for c, v in want.items():
        got = solver.wavefield(c)[sl]
        assert np.abs(got - v).max() < 2e-5 * scale, (c, v, got.min(), got.max())
    for c, v in V.items():
        assert np.abs(solver.wavefield(c)[sl] - v[sl]).max() < 1e-6 * np.abs(v).max(), c


def test_linear_velocity_one_step(oracle_built):
    from oracle import OracleSolver
    p = cases.uniform_box(ni=40, nj=40, nk=40, nt=2)
    V, G = _linear_fields(p)
    o = OracleSolver(p)
    for c, v in V.items():
        o.set_wavefield(c, v)
    o.run(1)
    check_linear_step(o, p, V, G)


def test_fault_below_strength_stays_locked(oracle_built):
    """Shear load 60 MPa under a strength of 0.65 x 100 MPa and no
    nucleation patch: the trial traction never reaches the friction law's
    bound, the fault never slips and the wavefield stays exactly zero."""
    from oracle import OracleSolver
    p = inputs.small_planar(nt=20)
    p.T0y[0][:] = 60.0e6
    o = OracleSolver(p)
    o.run(20)
    assert o.fault("Vs").max() <= 1e-12
    assert o.fault("Slip").max() == 0.0
    assert (o.fault("Init_t0") < 0).all()
    for c in ("Vx", "Vy", "Vz", "Txx", "Txy"):
        assert np.abs(o.wavefield(c)).max() == 0.0, c
    # the traction output stays the initial traction: Tn = -100 MPa, Ts1 = 60 MPa
    np.testing.assert_allclose(o.fault("Tn"), -100.0e6, rtol=1e-6)
    np.testing.assert_allclose(o.fault("Ts1"), 60.0e6, rtol=1e-6)


def test_locked_fault_matches_welded(oracle_built):
    """A velocity pulse crossing a fault that cannot slip (mu_s = 1000): the
    split-node solution keeps the velocity jump at zero and stays within a
    few percent of the same box without a fault (the difference is the
    lower-order one-sided operators next to the fault, and shrinks as the
    pulse widens)."""
    from oracle import OracleSolver
    res = {}
    for fault in (False, True):
        p = cases.uniform_box(fault=fault, ni=64, nj=48, nk=48, margin=4, nt=100)
        o = OracleSolver(p)
        g = cases.gaussian(p, (p.ni // 2 - 16, p.nj // 2, p.nk // 2), 500.0)
        o.set_wavefield("Vx", g)
        o.set_wavefield("Vy", 0.5 * g)
        o.run(90)
        res[fault] = {c: o.wavefield(c) for c in ("Vx", "Vy", "Txy")}
        if fault:
            vs = o.fault("Vs").max()
    # the pulse reached the fault
    assert np.abs(res[True]["Vx"][:, :, 32 + 4:]).max() > 0.02
    assert vs < 1e-6
    for c in res[False]:
        assert _rel(res[True][c], res[False][c]) < 0.03, c


def _sponge_mask_np(layer, vel, dt, nl, dh):
    """bdry_ablexp_cal_mask (src/forward/bdry_t.cu:704-722) restated in numpy
    float32, independently of the oracle's C++."""
    f = np.float32
    ln = f(nl) * f(dh)
    num_step = int(ln / f(vel) / f(dt))
    total = f(0.0)
    for n in range(num_step):
        total = f(total + f((f(n) * f(dt) * f(vel)) / ln) ** 2)
    alpha = f(0.6 / float(total))
    return float(np.exp(f(-alpha * f(f(layer) / f(nl)) ** 2)))


def test_sponge_masks_one_step(oracle_built):
    """One step from the same random state with and without the sponge: the
    ratio of the end levels is the mask, 1 outside the layers, the numpy
    mask formula inside (uniform 200 m grid), smallest at the outer face."""
    import dataclasses
    from oracle import OracleSolver
    L, vel = 6, 5000.0
    base = inputs.small_planar(nt=2, pml=0)
    spg = dataclasses.replace(base, ablexp_layers=((L, L), (L, L), (L, 0)),
                              ablexp_ref_vel=((vel, vel), (vel, vel), (vel, vel)))
    rng = np.random.default_rng(5)
    a, b = OracleSolver(base), OracleSolver(spg)
    for c in range(9):
        f = (rng.standard_normal((base.nk, base.nj, base.ni)) + 3.0).astype(np.float32)
        a.set_wavefield(c, f)
        b.set_wavefield(c, f)
    a.run(1)
    b.run(1)
    wa, wb = a.wavefield("Txx"), b.wavefield("Txx")
    ratio = wb / wa
    ni, nj, nk = base.ni, base.nj, base.nk
    jm, km = nj // 2, nk // 2
    mask = [_sponge_mask_np(L - i, vel, base.dt, L, 200.0) for i in range(L)]
    # x-left layers along one line through the middle of the y-z face
    np.testing.assert_allclose(ratio[km, jm, :L], mask, rtol=3e-6)
    np.testing.assert_allclose(ratio[km, jm, ni - L:], mask[::-1], rtol=3e-6)
    np.testing.assert_allclose(ratio[km, :L, ni // 2], mask, rtol=3e-6)
    np.testing.assert_allclose(ratio[:L, jm, ni // 2], mask, rtol=3e-6)
    assert mask[0] < mask[-1] < 1.0
    # no damping under the free top or inside the layers' inner faces
    inner = ratio[L:, L:nj - L, L:ni - L]
    assert np.array_equal(inner, np.ones_like(inner))
    # a corner point takes the smallest of its masks
    np.testing.assert_allclose(ratio[0, 0, 0], mask[0], rtol=3e-6)


def test_surface_peaks_against_numpy(oracle_built):
    """The oracle's peak surface motion (PG_calcu_gpu, src/forward/wav_t.cu:138-216)
    against the same maxima computed in numpy from the surface velocities of
    every step: peak |V| and components, peak |dV/dt|, and peak |D| of the
    trapezoid-rule displacement."""
    from oracle import OracleSolver
    p = inputs.small_planar(nt=20)
    o = OracleSolver(p)
    dt = np.float32(p.dt)
    prev = np.zeros((3, p.nj, p.ni), np.float32)
    disp = np.zeros((3, p.nj, p.ni), np.float64)
    pk = np.zeros((15, p.nj, p.ni), np.float64)
    for _ in range(20):
        o.run(1)
        v = np.stack([o.wavefield(c)[-1] for c in ("Vx", "Vy", "Vz")]).astype(np.float32)
        a = np.abs((v - prev) / dt)
        disp += 0.5 * (v + prev).astype(np.float64) * float(dt)
        d = disp.astype(np.float32)
        vals = [np.sqrt((v ** 2).sum(0)), np.sqrt((v[:2] ** 2).sum(0)), *np.abs(v),
                np.sqrt((a ** 2).sum(0)), np.sqrt((a[:2] ** 2).sum(0)), *a,
                np.sqrt((d ** 2).sum(0)), np.sqrt((d[:2] ** 2).sum(0)), *np.abs(d)]
        pk = np.maximum(pk, np.stack(vals))
        prev = v
    got = o.surface_peaks()
    assert got[0].max() > 0
    np.testing.assert_allclose(got, pk, rtol=2e-5, atol=1e-12 * float(np.abs(pk).max()))


def test_sponge_rupture_float_vs_double(oracle_built):
    """A rupture with the sponge boundary: the float32 oracle (the reference's
    arithmetic) against the float64 build, slip rate, slip and surface peaks."""
    import dataclasses
    from oracle import OracleSolver
    p = dataclasses.replace(inputs.small_planar(nt=40, pml=0), ablexp_layers=((6, 6), (6, 6), (6, 0)),
                            ablexp_ref_vel=((6000.0, 6000.0),) * 3)
    o32, o64 = OracleSolver(p), OracleSolver(p, double=True)
    o32.run(40)
    o64.run(40)
    assert o64.fault("Vs").max() > 0.1
    for f in ("Vs", "Slip", "Ts1"):
        assert _rel(o32.fault(f), o64.fault(f)) < 1e-4, f
    assert _rel(o32.surface_peaks(), o64.surface_peaks()) < 1e-4
