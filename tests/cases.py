"""Known-answer problem builders for the tests (uniform Cartesian boxes on
an imported grid, with or without a fault)."""
from __future__ import annotations

import numpy as np

from cgfd import GRID_IMPORT, Problem
import inputs


def uniform_box(ni=40, nj=40, nk=40, h=100.0, fault=False, locked=True, free_surface=0, pml=0,
                dt=0.005, nt=10, dynamic_method=2, margin=4):
    """Homogeneous box on an imported uniform grid x = (i - ni/2) h, y = (j - nj/2) h,
    z = (k - nk + 1) h.  With ``fault`` a vertical fault at i = ni/2 covering
    the whole plane; ``locked`` sets mu_s = 1000 everywhere so it never slips."""
    lam, mu, rho = inputs._homog(ni, nj, nk)
    xs = (np.arange(ni) - ni // 2) * h
    ys = (np.arange(nj) - nj // 2) * h
    zs = (np.arange(nk) - (nk - 1)) * h
    z3, y3, x3 = np.meshgrid(zs, ys, xs, indexing="ij")
    kw = {}
    if fault:
        fg = [1, nj, 1, nk]
        st = inputs._stress(nj, nk, fg, (nj // 2, nk // 2), 0, t_nuc=60.0)
        ms = st[3]
        if locked:
            ms = np.full_like(ms, 1000.0)
        kw = dict(fault_x_index=[ni // 2 + 1], fault_grid=[fg],
                  T0x=st[0][None], T0y=st[1][None], T0z=st[2][None], mu_s=ms[None],
                  mu_d=st[4][None], Dc=st[5][None], C0=st[6][None], welded_margin=margin)
    else:
        e = np.zeros((0, nk, nj), np.float32)
        kw = dict(fault_x_index=[], fault_grid=[], T0x=e, T0y=e, T0z=e, mu_s=e, mu_d=e, Dc=e, C0=e)
    P = ((pml, pml), (pml, pml), (pml, 0 if free_surface else pml))
    return Problem(ni=ni, nj=nj, nk=nk, dt=dt, lam=lam, mu=mu, rho=rho,
                   dynamic_method=dynamic_method, free_surface=free_surface, pml_layers=P,
                   pml_ref_vel=((6000.0, 6000.0),) * 3, grid_mode=GRID_IMPORT,
                   x3d=np.ascontiguousarray(x3, np.float32), y3d=np.ascontiguousarray(y3, np.float32),
                   z3d=np.ascontiguousarray(z3, np.float32), max_records=nt + 1,
                   name=f"uniform_box_{ni}x{nj}x{nk}", **kw)


def gaussian(prob, centre, width, h=100.0):
    """exp(-|x - centre|^2 / width^2) on the box's index grid, [nk, nj, ni]."""
    k, j, i = np.meshgrid(np.arange(prob.nk), np.arange(prob.nj), np.arange(prob.ni), indexing="ij")
    r2 = ((i - centre[0]) ** 2 + (j - centre[1]) ** 2 + (k - centre[2]) ** 2) * h * h
    return np.exp(-r2 / (width * width)).astype(np.float32)
