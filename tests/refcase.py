"""Runs of the reference's own solver on a Problem, for the parity tests.

oracle/_ref/cgfd_ref_main is hpc-lee/gpu-CGFD3D-dynamic's ``main``
(src/forward/main_curv_col_el_3d.cu) built from its unmodified sources by
oracle/build_ref.py against single-rank MPI and netCDF-classic stand-ins.
``write_reference_case`` writes a Problem as the reference's par JSON and
input files (par_files.write_case plus every key par_t.cu:64-900 reads, so
that nothing of the reference's parameter struct is left unset);
``run_reference`` runs the program on GPU 0; ``read_reference_outputs``
reads its fault netCDF file(s) and SAC traces.

Time base of the reference (drv_rk_curv_col.cu:209-636): with
number_of_time_steps = N it takes nt_total = N + 1 steps
(main_curv_col_el_3d.cu:483); before step it it samples the stations and
writes fault record it / io_time_skip, so record r holds the fault fields
after r * skip steps, and Peak_vs / Init_t0 are written after the last
step (io_fault_end_t_nc_put, drv_rk_curv_col.cu:644).
"""
from __future__ import annotations

import json
import os
import re
import subprocess

import numpy as np

import par_files

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "cgfd_ref_main")

# welded margin fixed in the reference (fault_info.cu:1044-1060)
REF_WELDED_MARGIN = 40


def reference_built():
    return os.path.exists(REF_EXE)


def write_reference_case(prob, case_dir, nt, medium="import", io_time_skip=1):
    """par.json + inputs of ``prob`` for the reference; returns the par path."""
    if prob.welded_margin != REF_WELDED_MARGIN:
        raise ValueError("the reference welds the 40 nodes next to the fault's edges; "
                         f"this problem asks for {prob.welded_margin}")
    names = [f"s{q}" for q in range(0 if prob.stations is None else len(prob.stations))]
    path = par_files.write_case(prob, case_dir, nt=nt, medium=medium, io_time_skip=io_time_skip,
                                station_names=names)
    par = json.load(open(path))
    out = par["output_dir"]
    par.pop("welded_margin", None)
    par.update({
        "number_of_mpiprocs_x": 1,
        "is_export_grid": 0, "grid_export_dir": out,
        "metric_calculation_method": {"calculate": 1},
        "is_export_metric": 0,
        "is_export_media": 0, "media_export_dir": out,
        "receiver_line": [],
        "slice": {"x_index": [], "y_index": [], "z_index": []},
        "snapshot": [],
        "check_nan_every_number_of_steps": 0,
        "output_all": 0,
    })
    if "in_station_file" not in par:
        par["in_station_file"] = os.path.join(case_dir, "no_stations.txt")
    if "fault_station_file" not in par:
        par["fault_station_file"] = os.path.join(case_dir, "no_fault_stations.txt")
    with open(path, "w") as fh:
        json.dump(par, fh, indent=2)
    return path


def run_reference(par_path, timeout=900):
    """Run the reference on GPU 0; returns (stdout, wall seconds of its time
    loop as it prints them)."""
    r = subprocess.run([REF_EXE, par_path, "0"], capture_output=True, text=True, timeout=timeout,
                       cwd=os.path.dirname(par_path))
    with open(os.path.join(os.path.dirname(par_path), "reference.log"), "w") as fh:
        fh.write(r.stdout + "\n---- stderr ----\n" + r.stderr)
    logdir = os.environ.get("CGFD_REF_LOGDIR")
    if logdir:
        os.makedirs(logdir, exist_ok=True)
        name = os.path.basename(os.path.dirname(par_path))
        with open(os.path.join(logdir, f"reference_{name}.log"), "w") as fh:
            fh.write(r.stdout[-200000:] + "\n---- stderr ----\n" + r.stderr[-50000:])
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed ({r.returncode}):\n{r.stdout[-3000:]}\n{r.stderr[-3000:]}")
    m = re.search(r"Runing Time of time :\s*([0-9.eE+-]+)", r.stdout)
    return r.stdout + r.stderr, (float(m.group(1)) if m else float("nan"))


def _sac_prefix(out, name):
    """File-name prefix of a station's traces.  The reference copies each
    station's name onto itself with sprintf (io_funcs.cu:244, :2262: source
    and destination are the same buffer when every station lies in the
    domain), which the C library leaves empty: every station then writes
    ".Vx.sac" etc., and the last one's traces are what remain."""
    return name if os.path.exists(os.path.join(out, f"{name}.Vx.sac")) or \
        os.path.exists(os.path.join(out, f"{name}.Vs.sac")) else ""


def read_reference_outputs(prob, par_path):
    """Fault files (one dict per fault), station traces [nsta, 9, nt_total]
    and fault-station traces [nfsta, 9, nt_total] of a finished run, with the
    indices of the stations those traces belong to (all of them, or only the
    last one when the reference wrote every station under an empty name)."""
    par = json.load(open(par_path))
    out = par["output_dir"]
    want = [f"fault_i{x}_px0_py0_pz0.nc" for x in prob.fault_x_index]
    nsta = 0 if prob.stations is None else len(prob.stations)
    if nsta and not _sac_prefix(out, "s0"):
        want.append(".Vx.sac")
    elif nsta:
        want += [f"s{q}.Vx.sac" for q in range(nsta)]
    missing = [w for w in want if not os.path.exists(os.path.join(out, w))]
    if missing:
        log = os.path.join(os.path.dirname(par_path), "reference.log")
        tail = open(log).read()[-4000:] if os.path.exists(log) else ""
        raise FileNotFoundError(f"reference outputs missing: {missing}; {out} holds {sorted(os.listdir(out))[:40]}; "
                                f"log tail:\n{tail}")
    faults = [par_files.read_fault_output(os.path.join(out, f"fault_i{x}_px0_py0_pz0.nc"))
              for x in prob.fault_x_index]
    def traces(n, prefix, names, cmps):
        if n == 0:
            return np.zeros((0, len(cmps), 0), np.float32), []
        if _sac_prefix(out, prefix + names[0]):
            idx = list(range(n))
            tr = [[par_files.read_sac(os.path.join(out, f"{prefix}{names[q]}.{c}.sac"))[3] for c in cmps] for q in idx]
        else:
            idx = [n - 1]
            tr = [[par_files.read_sac(os.path.join(out, f"{prefix}.{c}.sac"))[3] for c in cmps]]
        return np.array(tr, np.float32), idx
    sta, sta_idx = traces(nsta, "", [f"s{q}" for q in range(nsta)], par_files.CMP)
    nf = 0 if prob.fault_stations is None else len(prob.fault_stations)
    fsta, fsta_idx = traces(nf, "fault_", [f"f{q}" for q in range(nf)], par_files.FAULT_CMP)
    return faults, sta, fsta, sta_idx, fsta_idx
