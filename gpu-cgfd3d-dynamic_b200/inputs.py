"""Seeded synthetic inputs for the forward dynamic-rupture path.

The reference ships no input files: its examples generate them with MATLAB
scripts (example/tpv/prep_fault/conf_fault_grid.m: planar fault surface
x = 0, y = (j - nj/2) dh, z = (k - nk) dh; conf_fault_stress.m: mu_s = 1000
outside fault_grid, nucleation patch above strength).  These generators
restate that construction in numpy for the problem sizes this project
measures on, all in the reference's axes (x fault normal, y strike, z up):

* ``tpv_planar``   -- homogeneous half space, vertical planar fault, flat
  free surface, CFS-PML (the 160x100x80 case and scaled-down test cases);
* ``hills_layered`` -- curvilinear grid under Gaussian-hill topography,
  layered medium with a smoothed random perturbation, vertical fault
  (the 600x300x240 case the benchmark runs).

Every generator is deterministic for a given seed.
"""
from __future__ import annotations

import math

import numpy as np

from cgfd import GRID_FAULT_PLANE, GRID_IMPORT, Problem

MPA = 1.0e6


def _homog(ni, nj, nk, vp=6000.0, vs=3464.0, rho=2670.0):
    # md_gen_uniform_el_iso (src/forward/md_t.cu:378-417): products in
    # float, the subtraction of 2 mu in double
    vp32, vs32, rho32 = np.float32(vp), np.float32(vs), np.float32(rho)
    mu = vs32 * vs32 * rho32
    lam = np.float32(float(vp32 * vp32 * rho32) - 2.0 * float(mu))
    shape = (nk, nj, ni)
    return (np.full(shape, lam, np.float32), np.full(shape, mu, np.float32),
            np.full(shape, np.float32(rho), np.float32))


def _stress(nj, nk, fault_grid, nuc_center, nuc_half, tn=-100.0, ts=60.0, t_nuc=70.0,
            mu_s=0.65, mu_d=0.50, dc=0.30, c0=0.0, rng=None, ts_field=None):
    """Initial traction and friction on one fault [nk, nj] (0-based arrays,
    fault_grid 1-based inclusive like the par file)."""
    j1, j2, k1, k2 = [v - 1 for v in fault_grid]
    T0x = np.full((nk, nj), tn * MPA, np.float32)
    T0y = np.full((nk, nj), ts * MPA, np.float32) if ts_field is None else ts_field.astype(np.float32)
    T0z = np.zeros((nk, nj), np.float32)
    jc, kc = nuc_center
    T0y[kc - nuc_half:kc + nuc_half + 1, jc - nuc_half:jc + nuc_half + 1] = t_nuc * MPA
    ms = np.full((nk, nj), 1000.0, np.float32)
    ms[k1:k2 + 1, j1:j2 + 1] = mu_s
    md = np.full((nk, nj), mu_d, np.float32)
    Dc = np.full((nk, nj), dc, np.float32)
    C0 = np.full((nk, nj), c0, np.float32)
    return T0x, T0y, T0z, ms, md, Dc, C0


def tpv_planar(ni=100, nj=160, nk=80, h=200.0, fault_x_index=None, fault_grid=None,
               nuc_center=None, nuc_half=7, pml=10, dt=0.01, nt=600, nsta=8, seed=1000,
               margin=40, dynamic_method=2, free_surface=1, mu_s=0.65):
    """Homogeneous half space with a vertical planar fault.

    Defaults are the 160x100x80 case (h = 200 m, fault at x index 51,
    fault_grid [21, 141, 21, 80], 15x15-node nucleation patch at 70 MPa
    centred at strike node 81 and mid-depth of the fault, mu_s 0.65,
    mu_d 0.50, Dc 0.30 m, 10-layer CFS-PML on five faces, dt 0.01 s,
    600 steps, 8 surface stations)."""
    rng = np.random.default_rng(seed)
    if fault_x_index is None:
        fault_x_index = ni // 2 + 1
    if fault_grid is None:
        fault_grid = [int(round(nj * 0.125)) + 1, int(round(nj * 0.875)) + 1,
                      int(round(nk * 0.25)) + 1, nk]
    if nuc_center is None:
        jc = (fault_grid[0] + fault_grid[1]) // 2 - 1
        kc = nk - 1 - (nk - fault_grid[2] + 1) // 2
        nuc_center = (jc, kc)
    lam, mu, rho = _homog(ni, nj, nk)
    # conf_fault_grid.m with 1-based j, k
    jj, kk = np.meshgrid(np.arange(1, nj + 1), np.arange(1, nk + 1))
    fx = np.zeros((1, nk, nj), np.float32)
    fy = ((jj - nj / 2.0) * h).astype(np.float32)[None]
    fz = ((kk - nk) * h).astype(np.float32)[None]
    st = _stress(nj, nk, fault_grid, nuc_center, nuc_half, mu_s=mu_s)
    sta_i = rng.integers(pml + 2, ni - pml - 2, nsta)
    sta_j = rng.integers(pml + 2, nj - pml - 2, nsta)
    stations = np.stack([sta_i, sta_j, np.full(nsta, nk - 1)], 1).astype(np.float32)
    fsta = np.array([[nuc_center[0], nuc_center[1]],
                     [nuc_center[0] + nj // 8, nuc_center[1]],
                     [nuc_center[0], nk - 1]], np.float32)
    P = ((pml, pml), (pml, pml), (pml, 0 if free_surface else pml))
    vp = float(np.sqrt((lam[0, 0, 0] + 2 * mu[0, 0, 0]) / rho[0, 0, 0]))
    return Problem(ni=ni, nj=nj, nk=nk, dt=dt, lam=lam, mu=mu, rho=rho,
                   fault_x_index=[fault_x_index], fault_grid=[fault_grid],
                   T0x=st[0][None], T0y=st[1][None], T0z=st[2][None], mu_s=st[3][None],
                   mu_d=st[4][None], Dc=st[5][None], C0=st[6][None],
                   dynamic_method=dynamic_method, welded_margin=margin, free_surface=free_surface,
                   pml_layers=P, pml_ref_vel=((vp, vp),) * 3,
                   grid_mode=GRID_FAULT_PLANE, fault_interval=h,
                   fault_x=fx, fault_y=fy, fault_z=fz,
                   stations=stations, fault_stations=fsta, max_records=nt + 1,
                   name=f"tpv_planar_{nj}x{ni}x{nk}")


def _smooth(a, n):
    """Separable box smoothing with periodic wrap, n passes per axis."""
    out = a.astype(np.float64)
    for ax in range(out.ndim):
        for _ in range(n):
            out = (np.roll(out, 1, ax) + out + np.roll(out, -1, ax)) / 3.0
    return out


def hills_layered(ni=300, nj=600, nk=240, h=100.0, pml=20, seed=1001, nsta=32,
                  fault_len=400, fault_depth=180, margin=40, dynamic_method=2, nt=3000,
                  cfl=0.5, nhills=8, dip=None, vk_stress=False, nuc_half=7):
    """Curvilinear 600x300x240 case (x strike 600, y normal 300, z 240 in the
    task's axes; here ni = 300 normal, nj = 600 strike, nk = 240 up).

    Topography = sum of ``nhills`` Gaussian hills (amplitude U[100, 800] m,
    sigma U[2, 6] km); z is stretched linearly from the flat bottom to the
    surface.  Medium: four layers with Vs 2.0/2.6/3.1/3.6 km/s, Vp = 1.73 Vs,
    rho = 310 Vp^0.25 (Gardner), times (1 + 0.03 N(0,1)) smoothed.  Vertical
    fault at the x centre, fault_len x fault_depth nodes below the surface,
    friction as in ``tpv_planar``; 20-layer PML; dt = cfl * h / (sqrt(3) Vp_max).

    ``dip`` (degrees): the grid is sheared along x by depth * cot(dip), so
    the fault plane i = ni // 2 dips at that angle below the topography
    (dt then uses the sheared cell's point-to-plane distance
    h / sqrt(2 + (1 + cot dip)^2)).  ``vk_stress``: the shear traction is a
    von Karman field (correlation 2 km, Hurst 0.8, std 8 MPa, mean 60 MPa)
    kept 0.5 MPa below the static strength outside the nucleation patch.
    With a dip, the 100 MPa compression acts along the plane's normal."""
    rng = np.random.default_rng(seed)
    i0 = ni // 2                         # 0-based fault plane
    xs = (np.arange(ni) - i0) * h
    ys = (np.arange(nj) - nj / 2.0) * h
    X2, Y2 = np.meshgrid(xs, ys)         # [nj, ni]
    topo = np.zeros_like(X2)
    Lx, Ly = xs[-1] - xs[0], ys[-1] - ys[0]
    for _ in range(nhills):
        amp = rng.uniform(100.0, 800.0)
        sig = rng.uniform(2000.0, 6000.0)
        cx = rng.uniform(xs[0] + 0.2 * Lx, xs[-1] - 0.2 * Lx)
        cy = rng.uniform(ys[0] + 0.1 * Ly, ys[-1] - 0.1 * Ly)
        topo += amp * np.exp(-((X2 - cx) ** 2 + (Y2 - cy) ** 2) / (2 * sig * sig))
    zb = -(nk - 1) * h
    t = np.arange(nk) / (nk - 1.0)
    z3 = zb + (topo[None, :, :] - zb) * t[:, None, None]          # [nk, nj, ni]
    depth = topo[None] - z3
    if dip is None:
        x3 = np.broadcast_to(X2[None], (nk, nj, ni))
    else:
        x3 = (X2[None] + depth * (1.0 / math.tan(math.radians(dip)))).astype(np.float32)
    y3 = np.broadcast_to(Y2[None], (nk, nj, ni))
    bounds = [0.0, 2000.0, 6000.0, 12000.0]
    vs_l = [2000.0, 2600.0, 3100.0, 3600.0]
    vs = np.full(depth.shape, vs_l[0])
    for b, v in zip(bounds[1:], vs_l[1:]):
        vs = np.where(depth >= b, v, vs)
    pert = _smooth(rng.standard_normal((nk, nj, ni)), 3)
    pert = pert / max(pert.std(), 1e-12)
    vs = vs * (1.0 + 0.03 * pert)
    vp = 1.73 * vs
    rho = 310.0 * vp ** 0.25
    mu = (vs * vs * rho).astype(np.float32)
    lam = (vp * vp * rho - 2.0 * vs * vs * rho).astype(np.float32)
    vp_max = float(vp.max())
    del vs, vp, pert
    if dip is None:
        dt = cfl * h / (math.sqrt(3.0) * vp_max)
    else:
        cot = 1.0 / math.tan(math.radians(dip))
        dt = cfl * h / (math.sqrt(2.0 + (1.0 + cot) ** 2) * vp_max)
    dt = float(f"{dt:.3g}")
    jc = nj // 2
    fault_grid = [jc - fault_len // 2 + 1, jc + fault_len // 2, nk - fault_depth + 1, nk]
    kc = nk - 1 - fault_depth // 2
    ts_field = None
    if vk_stress:
        strength = 0.65 * 100.0
        ts_field = np.minimum(60.0 + 8.0 * von_karman(nj, nk, h, rng=rng), strength - 0.5) * MPA
    # with a dip, the topography tilts the local normal and the projected
    # traction: the patch is raised to 80 MPa so that it still nucleates
    st = _stress(nj, nk, fault_grid, (jc - 1, kc), nuc_half, ts_field=ts_field,
                 t_nuc=70.0 if dip is None else 80.0)
    if dip is not None:
        # compression of 100 MPa along the dipping plane's normal
        # (sin dip, 0, cos dip); the shear stays along strike (y)
        d = math.radians(dip)
        st = (np.full((nk, nj), -100.0 * MPA * math.sin(d), np.float32), st[1],
              np.full((nk, nj), -100.0 * MPA * math.cos(d), np.float32)) + tuple(st[3:])
    sta = np.stack([rng.integers(pml + 4, ni - pml - 4, nsta), rng.integers(pml + 4, nj - pml - 4, nsta),
                    np.full(nsta, nk - 1)], 1).astype(np.float32)
    fsta = np.array([[jc - 1, kc], [jc - 1 + fault_len // 4, kc], [jc - 1, nk - 1]], np.float32)
    P = ((pml, pml), (pml, pml), (pml, 0))
    vref = ((vp_max, vp_max),) * 3
    return Problem(ni=ni, nj=nj, nk=nk, dt=dt, lam=lam, mu=mu, rho=rho.astype(np.float32),
                   fault_x_index=[i0 + 1], fault_grid=[fault_grid],
                   T0x=st[0][None], T0y=st[1][None], T0z=st[2][None], mu_s=st[3][None],
                   mu_d=st[4][None], Dc=st[5][None], C0=st[6][None],
                   dynamic_method=dynamic_method, welded_margin=margin, free_surface=1,
                   pml_layers=P, pml_ref_vel=vref, grid_mode=GRID_IMPORT,
                   x3d=np.ascontiguousarray(x3, np.float32), y3d=np.ascontiguousarray(y3, np.float32),
                   z3d=np.ascontiguousarray(z3, np.float32),
                   stations=sta, fault_stations=fsta, max_records=nt + 1,
                   name=f"hills_layered_{nj}x{ni}x{nk}")


def small_planar(seed=7, dynamic_method=2, free_surface=1, pml=5, nt=60, **kw):
    """A 36x56x32 planar case with a 10-node welded margin: every feature of
    the path (split nodes reaching the free surface, PML on five faces, both
    x-operator directions) at a size the CPU oracle runs in seconds."""
    args = dict(ni=36, nj=56, nk=32, h=200.0, fault_x_index=18, fault_grid=[9, 48, 9, 32],
                nuc_center=(27, 22), nuc_half=3, pml=pml, dt=0.01, nt=nt, nsta=6, seed=seed,
                margin=10, dynamic_method=dynamic_method, free_surface=free_surface)
    args.update(kw)
    return tpv_planar(**args)


def von_karman(nj, nk, h, corr=2000.0, hurst=0.8, rng=None):
    """Zero-mean, unit-variance 2-D random field [nk, nj] with a von Karman
    spectrum P(k) ~ (1 + k^2 a^2)^-(H + 1) (correlation length a, Hurst
    exponent H), made by filtering white noise in the Fourier domain."""
    rng = np.random.default_rng() if rng is None else rng
    ky = 2.0 * np.pi * np.fft.fftfreq(nj, d=h)
    kz = 2.0 * np.pi * np.fft.fftfreq(nk, d=h)
    k2 = kz[:, None] ** 2 + ky[None, :] ** 2
    amp = (1.0 + k2 * corr * corr) ** (-(hurst + 1.0) / 2.0)
    f = np.real(np.fft.ifft2(np.fft.fft2(rng.standard_normal((nk, nj))) * amp))
    f -= f.mean()
    return f / max(f.std(), 1e-30)


def _hill_coords(ni, nj, nk, h, nhills, rng):
    """Curvilinear coordinates [nk, nj, ni] under a sum of Gaussian hills,
    stretched linearly from a flat bottom; the fault plane is x = 0 at
    i = ni // 2."""
    xs = (np.arange(ni) - ni // 2) * h
    ys = (np.arange(nj) - nj / 2.0) * h
    X2, Y2 = np.meshgrid(xs, ys)
    topo = np.zeros_like(X2)
    for _ in range(nhills):
        amp = rng.uniform(100.0, 800.0) * h / 100.0
        sig = rng.uniform(2000.0, 6000.0) * h / 100.0
        cx = rng.uniform(xs[0], xs[-1])
        cy = rng.uniform(ys[0], ys[-1])
        topo += amp * np.exp(-((X2 - cx) ** 2 + (Y2 - cy) ** 2) / (2 * sig * sig))
    zb = -(nk - 1) * h
    t = np.arange(nk) / (nk - 1.0)
    z3 = zb + (topo[None] - zb) * t[:, None, None]
    x3 = np.broadcast_to(X2[None], (nk, nj, ni))
    y3 = np.broadcast_to(Y2[None], (nk, nj, ni))
    return (np.ascontiguousarray(x3, np.float32), np.ascontiguousarray(y3, np.float32),
            np.ascontiguousarray(z3, np.float32))


def ensemble_scenarios(n=64, seed=1003, nt=1500, size_lo=(64, 96, 64), size_hi=(160, 256, 128),
                       pml=10, margin=10, cfl=0.5):
    """A seeded ensemble of rupture scenarios of uneven size (the batched
    workload): per scenario the grid (fault-normal ni in [64, 160], strike
    nj in [96, 256], depth nk in [64, 128]) and spacing h in [100, 200] m
    are drawn uniformly; the medium is homogeneous (6000 / 3464 m/s,
    2670 kg/m^3); the vertical fault at ni // 2 spans 75% of the strike and
    the top 75% of the depth; the shear traction is a von Karman field
    (correlation 2 km, Hurst 0.8, std 8 MPa, mean 60 MPa) kept below 95% of
    the static strength, with a 7 x 7-node nucleation patch at a random
    place raised 2 MPa above it; mu_s in [0.6, 0.7], mu_d 0.5, Dc in
    [0.2, 0.5] m; half of the scenarios have Gaussian-hill topography, the
    others a flat surface; 10-layer CFS-PML, free surface, dt at CFL 0.5."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        ni = int(rng.integers(size_lo[0], size_hi[0] + 1))
        nj = int(rng.integers(size_lo[1], size_hi[1] + 1))
        nk = int(rng.integers(size_lo[2], size_hi[2] + 1))
        h = float(rng.uniform(100.0, 200.0))
        mu_s = float(rng.uniform(0.6, 0.7))
        dc = float(rng.uniform(0.2, 0.5))
        hills = bool(rng.integers(0, 2))
        lam, mu, rho = _homog(ni, nj, nk)
        fg = [int(round(nj * 0.125)) + 1, int(round(nj * 0.875)) + 1, int(round(nk * 0.25)) + 1, nk]
        j1, j2, k1, k2 = [v - 1 for v in fg]
        strength = mu_s * 100.0
        ts = 60.0 + 8.0 * von_karman(nj, nk, h, rng=rng)
        ts = np.minimum(ts, 0.95 * strength)
        jc = int(rng.integers(max(j1 + margin + 4, 3), max(j2 - margin - 3, j1 + margin + 5)))
        kc = int(rng.integers(max(k1 + margin + 4, 3), max(nk - 5, k1 + margin + 5)))
        ts[kc - 3:kc + 4, jc - 3:jc + 4] = strength + 2.0
        st = _stress(nj, nk, fg, (jc, kc), 3, t_nuc=strength + 2.0, mu_s=mu_s, dc=dc,
                     ts_field=ts * MPA)
        P = ((pml, pml), (pml, pml), (pml, 0))
        vp = float(np.sqrt((lam[0, 0, 0] + 2 * mu[0, 0, 0]) / rho[0, 0, 0]))
        dt = float(f"{cfl * h / (math.sqrt(3.0) * vp):.3g}")
        sta = np.stack([rng.integers(pml + 2, ni - pml - 2, 4), rng.integers(pml + 2, nj - pml - 2, 4),
                        np.full(4, nk - 1)], 1).astype(np.float32)
        geo = {}
        if hills:
            x3, y3, z3 = _hill_coords(ni, nj, nk, h, int(rng.integers(1, 4)), rng)
            geo = dict(grid_mode=GRID_IMPORT, x3d=x3, y3d=y3, z3d=z3)
        else:
            jj, kk = np.meshgrid(np.arange(1, nj + 1), np.arange(1, nk + 1))
            geo = dict(grid_mode=GRID_FAULT_PLANE, fault_interval=h,
                       fault_x=np.zeros((1, nk, nj), np.float32),
                       fault_y=((jj - nj / 2.0) * h).astype(np.float32)[None],
                       fault_z=((kk - nk) * h).astype(np.float32)[None])
        out.append(Problem(ni=ni, nj=nj, nk=nk, dt=dt, lam=lam, mu=mu, rho=rho,
                           fault_x_index=[ni // 2 + 1], fault_grid=[fg],
                           T0x=st[0][None], T0y=st[1][None], T0z=st[2][None], mu_s=st[3][None],
                           mu_d=st[4][None], Dc=st[5][None], C0=st[6][None],
                           dynamic_method=2, welded_margin=margin, free_surface=1,
                           pml_layers=P, pml_ref_vel=((vp, vp),) * 3, stations=sta,
                           fault_stations=np.array([[jc, kc]], np.float32), max_records=nt + 1,
                           name=f"scenario_{q}_{nj}x{ni}x{nk}_{'hills' if hills else 'flat'}", **geo))
    return out


def two_faults(nt=60, dynamic_method=2, seed=9):
    """Two parallel vertical faults 14 nodes apart in a 44x64x32 planar grid
    (h = 200 m), each with its own fault_grid, nucleation patch and friction:
    the multi-fault path (one fault_coord / init_stress set per fault)."""
    ni, nj, nk, h = 44, 64, 32, 200.0
    lam, mu, rho = _homog(ni, nj, nk)
    fxi = [15, 29]
    grids = [[9, 56, 9, 32], [13, 52, 11, 32]]
    nucs = [((30, 22), 3), ((36, 20), 2)]
    jj, kk = np.meshgrid(np.arange(1, nj + 1), np.arange(1, nk + 1))
    fx = np.stack([np.zeros((nk, nj)), np.full((nk, nj), (fxi[1] - fxi[0]) * h)]).astype(np.float32)
    fy = np.stack([(jj - nj / 2.0) * h] * 2).astype(np.float32)
    fz = np.stack([(kk - nk) * h] * 2).astype(np.float32)
    sts = [_stress(nj, nk, g, c, r, mu_s=ms, dc=dc) for g, (c, r), ms, dc in
           zip(grids, nucs, (0.65, 0.62), (0.30, 0.25))]
    arr = lambda q: np.stack([st[q] for st in sts])
    rng = np.random.default_rng(seed)
    stations = np.stack([rng.integers(7, ni - 7, 4), rng.integers(7, nj - 7, 4), np.full(4, nk - 1)], 1).astype(np.float32)
    P = ((5, 5), (5, 5), (5, 0))
    vp = float(np.sqrt((lam[0, 0, 0] + 2 * mu[0, 0, 0]) / rho[0, 0, 0]))
    return Problem(ni=ni, nj=nj, nk=nk, dt=0.01, lam=lam, mu=mu, rho=rho, fault_x_index=fxi, fault_grid=grids,
                   T0x=arr(0), T0y=arr(1), T0z=arr(2), mu_s=arr(3), mu_d=arr(4), Dc=arr(5), C0=arr(6),
                   dynamic_method=dynamic_method, welded_margin=8, free_surface=1, pml_layers=P,
                   pml_ref_vel=((vp, vp),) * 3, grid_mode=GRID_FAULT_PLANE, fault_interval=h,
                   fault_x=fx, fault_y=fy, fault_z=fz, stations=stations,
                   fault_stations=np.array([[30, 22], [36, 20]], np.float32),
                   fault_station_fault=np.array([0, 1], np.int32), max_records=nt + 1, name="two_faults_64x44x32")
