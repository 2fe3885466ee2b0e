"""cgfd_run_fault_output: the fault records a run takes while it steps
(GPU).  Each record must equal what cgfd_get_fault_all returns at that
step of a plain run, bit for bit, for every fault, with and without an
output interval, and across calls."""
import numpy as np
import pytest

import inputs
from cgfd import CgfdError, Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("every", [1, 3])
def test_records_equal_plain_run(cgfd_lib, every):
    p = inputs.two_faults(nt=40)
    a, b = Solver(p), Solver(p)
    got = []
    for n in (7, 11):                      # two calls: the step index carries over
        got.append(b.run_fault_output(n, every))
    got = np.concatenate(got)
    want = []
    for it in range(18):
        if it % every == 0:
            want.append(np.stack([a.fault_all(f) for f in range(p.num_faults)]))
        a.run(1)
    want = np.array(want)
    assert got.shape == want.shape, (got.shape, want.shape)
    assert np.array_equal(got, want)
    assert a.steps_done == b.steps_done == 18
    for f in ("Vs", "Slip", "Init_t0"):
        assert np.array_equal(a.fault(f, 1), b.fault(f, 1))
    assert got[-1, 0, 3].max() > 0.1          # slip rate of fault 0 in the last record


def test_pinned_buffer_and_capacity(cgfd_lib):
    import torch
    p = inputs.small_planar(nt=20)
    s = Solver(p)
    rec = 11 * p.nk * p.nj
    buf = torch.empty(5 * rec, dtype=torch.float32, pin_memory=True)
    with pytest.raises(CgfdError, match="ERR_ARG"):
        s.run_fault_output(10, 2, out_ptr=buf.data_ptr(), max_records=4)   # 5 records needed
    assert s.steps_done == 0
    n = s.run_fault_output(10, 2, out_ptr=buf.data_ptr(), max_records=5)
    assert n == 5 and s.steps_done == 10
    ref = Solver(p)
    ref.run(8)
    assert np.array_equal(buf.numpy()[4 * rec:5 * rec].reshape(11, p.nk, p.nj), ref.fault_all(0))
