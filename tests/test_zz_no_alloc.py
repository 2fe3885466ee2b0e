"""cgfd_run_noalloc against cgfd_run (GPU).

The file name sorts last so that the suite also runs it after every other
test; it passes on its own as well.  Each test builds its own solvers."""
import numpy as np
import pytest

import inputs
from cgfd import CgfdError, Solver, WAVE_COMPONENTS

pytestmark = pytest.mark.gpu

TOL = 1e-6   # relative L2; the two entry points run the same kernels in the same order


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(np.asarray(b, np.float64)), 1e-30))


def _state(s, nfault):
    out = {}
    for fid in range(nfault):
        for f in ("Vs", "Slip", "Peak_vs", "Tn", "Ts1", "Init_t0"):
            out[(fid, f)] = s.fault(f, fid)
    for c in WAVE_COMPONENTS:
        out[c] = s.wavefield(c)
    out["stations"] = s.stations()
    out["fault_stations"] = s.fault_stations()
    return out


CASES = [("one fault", lambda m: inputs.small_planar(nt=40, dynamic_method=m), 1),
         # every fault of a solver takes its own slice of the shared array
         ("two faults", lambda m: inputs.two_faults(nt=40, dynamic_method=m), 2)]


@pytest.mark.parametrize("method", [1, 2])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_run_on_two_calls(cgfd_lib, case, method):
    _, make, nfault = case
    p = make(method)
    a, b = Solver(p), Solver(p)
    for call in range(2):
        a.run(9)
        b.run_noalloc(9)
        assert a.steps_done == b.steps_done == 9 * (call + 1)
        sa, sb = _state(a, nfault), _state(b, nfault)
        for k in sa:
            assert rel_l2(sb[k], sa[k]) <= TOL, (call, k, rel_l2(sb[k], sa[k]))
    for fid in range(nfault):
        assert a.fault("Vs", fid).max() > 0.1


def test_noalloc_allocates_no_device_memory(cgfd_lib):
    import torch
    p = inputs.small_planar(nt=30)
    s = Solver(p)
    s.run_noalloc(2)              # first call on the device: address look-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    s.run_noalloc(8)
    s.run_noalloc(8)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def _parallel_faults(nf, nj=200, nk=150, h=200.0, margin=4):
    """nf vertical planar faults 14 nodes apart, each over the whole plane
    (welded only within `margin` nodes of the sides and the bottom), loaded
    below strength: a split box of (nj - 2 margin) x (nk - margin) nodes."""
    ni = 14 * nf + 16
    lam, mu, rho = inputs._homog(ni, nj, nk)
    fxi = [9 + 14 * q for q in range(nf)]
    jj, kk = np.meshgrid(np.arange(1, nj + 1), np.arange(1, nk + 1))
    fx = np.stack([np.full((nk, nj), (x - fxi[0]) * h) for x in fxi]).astype(np.float32)
    fy = np.stack([(jj - nj / 2.0) * h] * nf).astype(np.float32)
    fz = np.stack([(kk - nk) * h] * nf).astype(np.float32)
    grid = [1, nj, 1, nk]
    st = inputs._stress(nj, nk, grid, (nj // 2, nk - 10), 2, t_nuc=60.0)
    arr = lambda q: np.stack([st[q]] * nf)
    return inputs.Problem(ni=ni, nj=nj, nk=nk, dt=0.01, lam=lam, mu=mu, rho=rho, fault_x_index=fxi,
                          fault_grid=[grid] * nf, T0x=arr(0), T0y=arr(1), T0z=arr(2), mu_s=arr(3), mu_d=arr(4),
                          Dc=arr(5), C0=arr(6), welded_margin=margin, free_surface=1,
                          grid_mode=inputs.GRID_FAULT_PLANE, fault_interval=h, fault_x=fx, fault_y=fy, fault_z=fz,
                          stations=np.array([[4, 10, nk - 1]], np.float32), max_records=8,
                          name=f"parallel_faults_{nf}")


def test_noalloc_rejects_faults_whose_sum_exceeds_the_scratch(cgfd_lib):
    # each split box is 192 x 146 nodes: 108 * 198 * 152 floats = 3.1 Mi;
    # two faults (6.2 Mi together) fit the 8 Mi array, three (9.3 Mi) do not
    ok = Solver(_parallel_faults(2))
    ok.run_noalloc(1)
    assert ok.steps_done == 1
    s = Solver(_parallel_faults(3))
    with pytest.raises(CgfdError, match="ERR_ARG.*scratch floats together"):
        s.run_noalloc(1)
    assert s.steps_done == 0


def test_noalloc_rejects_a_fault_beyond_the_scratch(cgfd_lib):
    # split box 492 x 196 nodes: 108 * 498 * 202 floats > 8 Mi
    p = inputs.tpv_planar(ni=24, nj=500, nk=200, fault_x_index=12, fault_grid=[1, 500, 1, 200], margin=4,
                          pml=0, nuc_half=2, nsta=2, nt=4)
    s = Solver(p)
    with pytest.raises(CgfdError, match="ERR_ARG.*scratch"):
        s.run_noalloc(1)
    assert s.steps_done == 0
    s.run(1)                       # the solver is untouched and still runs
    assert s.steps_done == 1
