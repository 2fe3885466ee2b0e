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


def _state(s):
    out = {f: s.fault(f) for f in ("Vs", "Slip", "Peak_vs", "Tn", "Ts1", "Init_t0")}
    for c in WAVE_COMPONENTS:
        out[c] = s.wavefield(c)
    out["stations"] = s.stations()
    return out


@pytest.mark.parametrize("method", [1, 2])
def test_noalloc_matches_run_on_two_calls(cgfd_lib, method):
    p = inputs.small_planar(nt=40, dynamic_method=method)
    a, b = Solver(p), Solver(p)
    for call in range(2):
        a.run(9)
        b.run_noalloc(9)
        assert a.steps_done == b.steps_done == 9 * (call + 1)
        sa, sb = _state(a), _state(b)
        for k in sa:
            assert rel_l2(sb[k], sa[k]) <= TOL, (call, k, rel_l2(sb[k], sa[k]))
    assert a.fault("Vs").max() > 0.1


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
