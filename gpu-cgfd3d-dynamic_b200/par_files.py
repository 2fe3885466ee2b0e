"""Write a Problem as the reference's input files, and read the outputs.

The reference's users prepare a run with MATLAB scripts that write
fault_coord_<id>.nc (x, y, z [nk][nj]) and init_stress_<id>.nc (Tx, Ty, Tz,
mu_s, mu_d, Dc, C0 [nk][nj]) (example/tpv/prep_fault/conf_fault_grid.m,
conf_fault_stress.m), a station list, a fault-station list and the par JSON
file.  ``write_case`` produces the same set from a ``Problem`` for the
``cgfd_run`` driver; ``read_fault_output`` and ``read_sac`` read what the
driver writes.  netCDF classic I/O uses scipy.io.netcdf_file.
"""
from __future__ import annotations

import json
import os

import numpy as np

from cgfd import GRID_FAULT_PLANE, GRID_IMPORT, Problem

CMP = ("Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Tyz", "Txz", "Txy")
FAULT_CMP = ("Tn", "Ts1", "Ts2", "Vs", "Vs1", "Vs2", "Slip", "Slip1", "Slip2")


def _nc_write(path, dims, variables, version=1):
    from scipy.io import netcdf_file
    with netcdf_file(path, "w", version=version) as f:
        for name, n in dims:
            f.createDimension(name, n)
        for name, dnames, arr in variables:
            v = f.createVariable(name, arr.dtype, dnames)
            v[:] = arr


def write_case(prob: Problem, case_dir: str, nt: int, output_dir: str = None, io_time_skip: int = 1,
               medium: str = "import", station_names=None):
    """Write par.json and the input files of ``prob`` into ``case_dir``;
    returns the par file's path.  ``medium``: "import" writes the medium to
    media_px0_py0_pz0.nc, "code" relies on the driver's uniform medium
    (6000 / 3464 m/s, 2670 kg/m^3)."""
    os.makedirs(case_dir, exist_ok=True)
    out = output_dir or os.path.join(case_dir, "output")
    os.makedirs(out, exist_ok=True)
    nf = prob.num_faults
    par = {"number_of_total_grid_points_x": prob.ni, "number_of_total_grid_points_y": prob.nj,
           "number_of_total_grid_points_z": prob.nk, "number_of_mpiprocs_y": 1, "number_of_mpiprocs_z": 1,
           "size_of_time_step": float(prob.dt), "number_of_time_steps": int(nt), "time_start": 0.0,
           "time_check_stability": int(prob.check_stability), "io_time_skip": int(io_time_skip),
           "dynamic_method": int(prob.dynamic_method),
           "fault_x_index": [int(x) for x in prob.fault_x_index],
           "fault_grid": [int(v) for g in prob.fault_grid for v in g],
           "output_dir": out}
    names = [("boundary_x_left", 0, 0), ("boundary_x_right", 0, 1), ("boundary_y_front", 1, 0),
             ("boundary_y_back", 1, 1), ("boundary_z_bottom", 2, 0), ("boundary_z_top", 2, 1)]
    for key, d, s in names:
        if d == 2 and s == 1 and prob.free_surface:
            par[key] = {"free": "timg"}
        elif prob.ablexp_layers[d][s] > 0:
            par[key] = {"ablexp": {"number_of_layers": int(prob.ablexp_layers[d][s]),
                                   "ref_vel": float(prob.ablexp_ref_vel[d][s])}}
        elif prob.pml_layers[d][s] > 0:
            par[key] = {"cfspml": {"number_of_layers": int(prob.pml_layers[d][s]),
                                   "alpha_max": float(prob.pml_alpha_max[d][s]),
                                   "beta_max": float(prob.pml_beta_max[d][s]),
                                   "ref_vel": float(prob.pml_ref_vel[d][s])}}
    if prob.welded_margin != 40:
        # an extension key of cgfd_run (the reference fixes the margin at 40)
        par["welded_margin"] = int(prob.welded_margin)
    stress_dir = os.path.join(case_dir, "init_stress")
    os.makedirs(stress_dir, exist_ok=True)
    for f in range(nf):
        _nc_write(os.path.join(stress_dir, f"init_stress_{f + 1}.nc"), [("k", prob.nk), ("j", prob.nj)],
                  [(n, ("k", "j"), np.ascontiguousarray(a[f], np.float32)) for n, a in
                   (("Tx", prob.T0x), ("Ty", prob.T0y), ("Tz", prob.T0z), ("mu_s", prob.mu_s),
                    ("mu_d", prob.mu_d), ("Dc", prob.Dc), ("C0", prob.C0))])
    if prob.grid_mode == GRID_FAULT_PLANE:
        geo_dir = os.path.join(case_dir, "fault_coord")
        os.makedirs(geo_dir, exist_ok=True)
        for f in range(nf):
            _nc_write(os.path.join(geo_dir, f"fault_coord_{f + 1}.nc"), [("k", prob.nk), ("j", prob.nj)],
                      [(n, ("k", "j"), np.ascontiguousarray(a[f], np.float32)) for n, a in
                       (("x", prob.fault_x), ("y", prob.fault_y), ("z", prob.fault_z))])
        par["grid_generation_method"] = {"fault_plane": {"fault_geometry_dir": geo_dir,
                                                         "fault_init_stress_dir": stress_dir,
                                                         "fault_inteval": float(prob.fault_interval)}}
    else:
        geo_dir = os.path.join(case_dir, "grid")
        os.makedirs(geo_dir, exist_ok=True)
        _nc_write(os.path.join(geo_dir, "coord_px0_py0_pz0.nc"), [("k", prob.nk), ("j", prob.nj), ("i", prob.ni)],
                  [(n, ("k", "j", "i"), np.ascontiguousarray(a, np.float32)) for n, a in
                   (("x", prob.x3d), ("y", prob.y3d), ("z", prob.z3d))], version=2)
        par["grid_generation_method"] = {"grid_import": {"import_dir": geo_dir, "fault_init_stress_dir": stress_dir}}
    if medium == "import":
        md_dir = os.path.join(case_dir, "media")
        os.makedirs(md_dir, exist_ok=True)
        _nc_write(os.path.join(md_dir, "media_px0_py0_pz0.nc"), [("k", prob.nk), ("j", prob.nj), ("i", prob.ni)],
                  [(n, ("k", "j", "i"), np.ascontiguousarray(a, np.float32)) for n, a in
                   (("lambda", prob.lam), ("mu", prob.mu), ("rho", prob.rho))], version=2)
        par["medium"] = {"type": "elastic_iso", "input_way": "import", "import": md_dir}
    else:
        par["medium"] = {"type": "elastic_iso", "input_way": "code"}
    if prob.stations is not None and len(prob.stations):
        path = os.path.join(case_dir, "stations.txt")
        names = station_names or [f"s{q}" for q in range(len(prob.stations))]
        with open(path, "w") as fh:
            fh.write("# name flag_coord flag_depth x y z (grid indices from 1)\n")
            fh.write(f"{len(prob.stations)}\n")
            for n, (i, j, k) in zip(names, prob.stations):
                fh.write(f"{n} 0 0 {i + 1:.6f} {j + 1:.6f} {k + 1:.6f}\n")
        par["in_station_file"] = path
    if prob.fault_stations is not None and len(prob.fault_stations):
        path = os.path.join(case_dir, "fault_stations.txt")
        fid = prob.fault_station_fault if prob.fault_station_fault is not None else np.zeros(len(prob.fault_stations))
        with open(path, "w") as fh:
            fh.write(f"{len(prob.fault_stations)}\n")
            for q, ((j, k), f) in enumerate(zip(prob.fault_stations, fid)):
                fh.write(f"f{q} {int(f) + 1} {j + 1:.6f} {k + 1:.6f}\n")
        par["fault_station_file"] = path
    path = os.path.join(case_dir, "par.json")
    with open(path, "w") as fh:
        json.dump(par, fh, indent=2)
    return path


def read_fault_output(path):
    """dict of the fault output file's variables (numpy copies)."""
    from scipy.io import netcdf_file
    with netcdf_file(path, "r", mmap=False) as f:
        out = {k: np.array(v[:]) for k, v in f.variables.items()}
        out["_attrs"] = dict(f._attributes)
    return out


def read_surface_peaks(path):
    """dict of the PG_V_A_D file's variables [ny][nx] (ghost-inclusive) and
    its global attributes under "_attrs"."""
    return read_fault_output(path)


def read_sac(path):
    """(header floats [70], header ints [40], header chars [192], data) of a
    SAC file in native byte order."""
    raw = open(path, "rb").read()
    fh = np.frombuffer(raw[:280], np.float32)
    ih = np.frombuffer(raw[280:440], np.int32)
    kh = raw[440:632]
    data = np.frombuffer(raw[632:], np.float32)
    return fh, ih, kh, data
