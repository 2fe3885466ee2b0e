"""The reference's own arithmetic against the oracle and the CUDA path (GPU).

oracle/_ref/cgfd_ref_main is hpc-lee/gpu-CGFD3D-dynamic's unmodified solver
(src/forward/*.cu, src/lib/*.cu, src/media/*.cpp), built by
oracle/build_ref.py for sm_100a against single-rank MPI and netCDF-classic
stand-ins.  Each case writes a Problem as the reference's par JSON and input
files, runs the reference on GPU 0, and compares what it writes (the fault
netCDF file's records, Peak_vs and Init_t0, the station and fault-station
SAC traces, the surface peaks) with the oracle's and the CUDA path's values
for the same steps.  This pins the oracle: every other parity test compares
the CUDA path with the oracle.

Tolerance: relative L2 <= 1e-4 on slip rate, slip, peak slip rate,
tractions and station velocities; the rupture time of every node within one
time step and the same set of ruptured nodes.  The reference takes
number_of_time_steps + 1 steps (refcase.py); fault record r holds the fields
after r steps.
"""
import os

import numpy as np
import pytest

import inputs
import par_files
import refcase

pytestmark = pytest.mark.gpu

TOL = 1e-4
# fault fields compared record by record; Ts2, Vs2, Slip2 (the dip
# components of a strike-slip rupture) are compared against the norm of the
# strike component, since their own norm is at rounding level
FIELDS = ("Tn", "Ts1", "Vs", "Vs1", "Slip", "Slip1")
DIP_FIELDS = (("Ts2", "Ts1"), ("Vs2", "Vs1"), ("Slip2", "Slip1"))


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _needs_reference():
    if not refcase.reference_built():
        pytest.fail("oracle/_ref/cgfd_ref_main is not built: run oracle/build_ref.py "
                    "(__graft_entry__.build() does) where the reference tree is present")


def _cases():
    return {
        # the 160x100x80 planar case (h = 200 m, 10-layer CFS-PML on five
        # faces, flat free surface, 8 stations), both dynamic methods
        "planar_m2": (lambda: _with_fault_stations(inputs.tpv_planar(dynamic_method=2)), 600, "code", 100),
        "planar_m1": (lambda: _with_fault_stations(inputs.tpv_planar(dynamic_method=1)), 300, "code", 100),
        # curvilinear grid under hills (grid import) and a layered, perturbed
        # medium (media import)
        "hills": (lambda: inputs.hills_layered(ni=64, nj=160, nk=96, h=100.0, pml=10, nsta=6, fault_len=110,
                                               fault_depth=80, margin=40, nt=240, nhills=3), 240, "import", 60),
        # exponential sponge on five faces instead of the CFS-PML
        "sponge": (lambda: _sponge(inputs.tpv_planar(ni=60, nj=120, nk=64, pml=0, nsta=4, nt=200,
                                                     fault_grid=[21, 100, 21, 64])), 200, "code", 50),
    }


def _with_fault_stations(p):
    jc = (p.fault_grid[0][0] + p.fault_grid[0][1]) // 2 - 1
    p.fault_stations = np.array([[jc, p.nk - 20], [jc + 20.5, p.nk - 10.25]], np.float32)
    p.fault_station_fault = np.zeros(2, np.int32)
    return p


def _sponge(p):
    import dataclasses
    return dataclasses.replace(p, ablexp_layers=((10, 10), (10, 10), (10, 0)),
                               ablexp_ref_vel=((6000.0, 6000.0),) * 3)


_RUNS = {}


def _reference_run(name, tmp_root):
    """Run the reference once per case and session."""
    if name not in _RUNS:
        make, nt, medium, _ = _cases()[name]
        p = make()
        p.max_records = nt + 1
        case = os.path.join(tmp_root, name)
        par = refcase.write_reference_case(p, case, nt=nt, medium=medium)
        log, secs = refcase.run_reference(par)
        faults, sta, fsta, sta_idx, fsta_idx = refcase.read_reference_outputs(p, par)
        pg = None
        if p.free_surface:
            out = os.path.dirname(par) + "/output"
            pg = par_files.read_surface_peaks(os.path.join(out, "PG_V_A_D_px0_py0_pz0.nc"))
        _RUNS[name] = dict(p=p, nt=nt, faults=faults, sta=sta, fsta=fsta, sta_idx=sta_idx, fsta_idx=fsta_idx,
                           pg=pg, log=log, secs=secs)
    return _RUNS[name]


@pytest.fixture(scope="module")
def ref_root(tmp_path_factory):
    return str(tmp_path_factory.mktemp("reference_runs"))


def _check_solver(solver, R, every, label):
    """Fault records every `every` steps, then the end-of-run fields and
    traces after nt + 1 steps, of `solver` against the reference run R."""
    p, nt, F = R["p"], R["nt"], R["faults"][0]
    done = 0
    for rec in list(range(every, nt + 1, every)) + ([nt] if nt % every else []):
        solver.run(rec - done)
        done = rec
        for f in FIELDS:
            e = rel_l2(solver.fault(f), F[f][rec])
            assert e <= TOL, (label, rec, f, e)
        for f, ref_f in DIP_FIELDS:
            e = np.linalg.norm(solver.fault(f).astype(np.float64) - F[f][rec]) / max(
                np.linalg.norm(F[ref_f][rec].astype(np.float64)), 1e-30)
            assert e <= TOL, (label, rec, f, e)
    solver.run(1)                                   # the reference's step N + 1
    assert rel_l2(solver.fault("Peak_vs"), F["Peak_vs"]) <= TOL, label
    t0s, t0r = solver.fault("Init_t0"), F["Init_t0"]
    rup = t0r > 0
    assert rup.sum() > 100, (label, "no rupture in the reference run")
    assert np.array_equal(t0s > 0, rup), label
    assert np.abs(t0s[rup] - t0r[rup]).max() <= p.dt * 1.0001, label
    seis = solver.stations()[R["sta_idx"]]
    assert seis.shape == R["sta"].shape, (label, seis.shape, R["sta"].shape)
    assert rel_l2(seis[:, :3], R["sta"][:, :3]) <= TOL, (label, "station velocity")
    assert rel_l2(seis[:, 3:], R["sta"][:, 3:]) <= TOL, (label, "station stress")
    if len(R["fsta"]):
        fs = solver.fault_stations()[R["fsta_idx"]]
        for c, name in enumerate(par_files.FAULT_CMP):
            if name in ("Ts2", "Vs2", "Slip2"):
                continue
            mine, ref = fs[:, c], R["fsta"][:, c]
            if name in ("Vs", "Vs1", "Slip", "Slip1") and np.abs(ref).max() < 1e-6 and np.abs(mine).max() < 1e-6:
                # a node the rupture has not reached: slip rate and slip are
                # rounding noise of a zero velocity jump in both runs
                continue
            assert rel_l2(mine, ref) <= TOL, (label, "fault station", name)
    if R["pg"] is not None:
        from cgfd import PEAK_FIELDS
        mine = solver.surface_peaks()
        for c, name in enumerate(PEAK_FIELDS):
            ref = R["pg"][name][3:-3, 3:-3]
            assert rel_l2(mine[c], ref) <= TOL, (label, name, rel_l2(mine[c], ref))


@pytest.mark.parametrize("name", ["planar_m2", "planar_m1", "hills", "sponge"])
def test_cuda_path_matches_reference(cgfd_lib, ref_root, name):
    _needs_reference()
    from cgfd import Solver
    R = _reference_run(name, ref_root)
    _check_solver(Solver(R["p"]), R, _cases()[name][3], "cuda")


@pytest.mark.parametrize("name", ["planar_m2", "planar_m1", "hills", "sponge"])
def test_oracle_matches_reference(oracle_built, ref_root, name):
    _needs_reference()
    from oracle import OracleSolver
    R = _reference_run(name, ref_root)
    _check_solver(OracleSolver(R["p"]), R, _cases()[name][3], "oracle")


@pytest.mark.parametrize("name", ["planar_m2", "hills"])
def test_driver_files_match_reference(cgfd_lib, ref_root, name):
    """The drop-in: the same par.json given to the reference's ``main`` and
    to this project's ``cgfd_run`` gives the same files (fault netCDF records,
    Peak_vs and Init_t0, station SAC traces)."""
    import json
    import subprocess
    _needs_reference()
    R = _reference_run(name, ref_root)
    case = os.path.join(ref_root, name)
    par = json.load(open(os.path.join(case, "par.json")))
    out = os.path.join(case, "output_cgfd_run")
    os.makedirs(out, exist_ok=True)
    par["output_dir"] = out
    mine = os.path.join(case, "par_cgfd_run.json")
    with open(mine, "w") as fh:
        json.dump(par, fh)
    exe = os.path.join(os.path.dirname(cgfd_lib._name), "cgfd_run")
    r = subprocess.run([exe, mine, "0"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    p = R["p"]
    for fi, x in enumerate(p.fault_x_index):
        d = par_files.read_fault_output(os.path.join(out, f"fault_i{x}_px0_py0_pz0.nc"))
        ref = R["faults"][fi]
        assert d["Tn"].shape == ref["Tn"].shape
        np.testing.assert_allclose(d["time"], ref["time"], rtol=1e-6)
        for f in FIELDS:
            for rec in range(0, ref[f].shape[0], 20):
                assert rel_l2(d[f][rec], ref[f][rec]) <= TOL or np.linalg.norm(ref[f][rec]) == 0, (f, rec)
        for f in ("Peak_vs", "Init_t0"):
            assert d[f].shape == ref[f].shape
        assert rel_l2(d["Peak_vs"], ref["Peak_vs"]) <= TOL
        assert np.array_equal(d["Init_t0"] > 0, ref["Init_t0"] > 0)
    # station traces: this driver names them after the stations; the
    # reference's files of the stations it kept (refcase._sac_prefix)
    for k, q in enumerate(R["sta_idx"]):
        v = np.array([par_files.read_sac(os.path.join(out, f"s{q}.{c}.sac"))[3] for c in par_files.CMP])
        assert v.shape == R["sta"][k].shape, (q, v.shape, R["sta"][k].shape)
        assert rel_l2(v[:3], R["sta"][k][:3]) <= TOL, q
