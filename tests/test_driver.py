"""The par-file driver (gpu-cgfd3d-dynamic_b200/lib/cgfd_run).

CPU: its netCDF classic reader and writer against scipy's independent
implementation of the format, its SAC header layout, the JSON reader.
GPU: a whole run from par.json and reference-format input files, whose
output files must hold what the library returns for the same problem."""
import dataclasses
import json
import os
import subprocess

import numpy as np
import pytest

import inputs
import par_files

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER_DIR = os.path.join(ROOT, "gpu-cgfd3d-dynamic_b200", "driver")


@pytest.fixture(scope="module")
def io_check(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("io") / "driver_io_check")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-o", exe, os.path.join(ROOT, "tests", "driver_io_check.cpp"),
                           os.path.join(DRIVER_DIR, "ncclassic.cpp"), os.path.join(DRIVER_DIR, "sac.cpp")])
    return exe


def _floats(out):
    return np.array([float(x) for x in out.split()], np.float64).astype(np.float32)


@pytest.mark.parametrize("version", [1, 2])
def test_netcdf_reader_against_scipy(io_check, tmp_path, version):
    from scipy.io import netcdf_file
    path = str(tmp_path / f"in_v{version}.nc")
    rng = np.random.default_rng(version)
    a = rng.standard_normal((5, 7)).astype(np.float32)
    b = rng.standard_normal((3, 4, 6)).astype(np.float64)
    r = rng.standard_normal((4, 2, 3)).astype(np.float32)
    with netcdf_file(path, "w", version=version) as f:
        f.createDimension("time", None)
        for n, d in (("k", 5), ("j", 7), ("z", 3), ("y", 4), ("x", 6), ("b", 2), ("c", 3)):
            f.createDimension(n, d)
        f.title = "test"
        f.createVariable("a", "f4", ("k", "j"))[:] = a
        v = f.createVariable("bb", "f8", ("z", "y", "x"))
        v.units = "m"
        v[:] = b
        f.createVariable("rec", "f4", ("time", "b", "c"))[:] = r
        f.createVariable("t", "f4", ("time",))[:] = np.arange(4, dtype=np.float32)
    out = subprocess.run([io_check, "read", path, "a"], capture_output=True, text=True, check=True).stdout
    whole, slab = out.split("slab")
    np.testing.assert_array_equal(_floats(whole), a.ravel())
    np.testing.assert_array_equal(_floats(slab), a[1:, 1:3].ravel())
    out = subprocess.run([io_check, "read", path, "bb"], capture_output=True, text=True, check=True).stdout
    np.testing.assert_allclose(_floats(out), b.astype(np.float32).ravel(), rtol=0)
    out = subprocess.run([io_check, "read", path, "rec"], capture_output=True, text=True, check=True).stdout
    np.testing.assert_array_equal(_floats(out), r.ravel())
    out = subprocess.run([io_check, "read", path, "t"], capture_output=True, text=True, check=True).stdout
    np.testing.assert_array_equal(_floats(out), np.arange(4))


def test_netcdf_writer_read_by_scipy(io_check, tmp_path):
    path = str(tmp_path / "out.nc")
    subprocess.check_call([io_check, "write", path])
    d = par_files.read_fault_output(path)
    np.testing.assert_array_equal(d["time"], [0.0, 0.5])
    for rec in range(2):
        np.testing.assert_array_equal(d["Tn"][rec].ravel(), 100.0 * rec + np.arange(12))
        np.testing.assert_array_equal(d["Vs"][rec].ravel(), -np.arange(12) - rec)
    np.testing.assert_array_equal(d["Peak_vs"].ravel(), 0.25 * np.arange(12))
    assert d["Tn"].shape == (2, 3, 4) and d["Peak_vs"].shape == (3, 4)
    assert int(np.ravel(d["_attrs"]["i_index_with_ghosts_in_this_thread"])[0]) == 53
    assert list(np.ravel(d["_attrs"]["coords_of_mpi_topo"])) == [0, 0, 0]


def test_sac_header(io_check, tmp_path):
    path = str(tmp_path / "x.sac")
    subprocess.check_call([io_check, "sac", path])
    fh, ih, kh, data = par_files.read_sac(path)
    assert os.path.getsize(path) == 632 + 5 * 4
    np.testing.assert_array_equal(data, [1, 2, 3, 4, 5])
    assert fh[0] == np.float32(0.01) and fh[5] == 0.0 and fh[6] == np.float32(0.01) * 4
    assert (fh[31], fh[32], fh[33], fh[34]) == (1.5, 2.5, -3.5, np.float32(0.01))   # stla stlo stel stdp
    assert fh[35] == fh[36] == fh[37] == fh[38] == 0.0 and fh[57] == fh[58] == 0.0
    assert fh[1] == -12345.0 and fh[69] == -12345.0
    assert ih[6] == 6 and ih[9] == 5 and ih[15] == 1 and ih[35] == 1        # nvhdr npts iftype leven
    assert ih[0] == -12345 and ih[36] == -12345
    assert kh[:8] == b"-12345\0\0" and kh[160:168] == b"-12345\0\0"        # kstnm, kcmpnm
    assert kh[8:24] == b"-12345  " + b"\0" * 8 and kh[24:32] == b"-12345  "


def _driver():
    return os.path.join(ROOT, "gpu-cgfd3d-dynamic_b200", "lib", "cgfd_run")


@pytest.mark.gpu
@pytest.mark.parametrize("medium,case", [("import", "planar"), ("code", "hills"), ("import", "two_faults"),
                                         ("import", "sponge")])
def test_driver_run_matches_library(cgfd_lib, tmp_path, medium, case):
    from cgfd import PEAK_FIELDS, Solver
    nt, skip = 30, 3
    if case == "two_faults":
        p = inputs.two_faults(nt=nt)
    elif case == "hills":
        p = inputs.hills_layered(ni=48, nj=72, nk=40, h=100.0, pml=8, nsta=4, fault_len=48, fault_depth=30,
                                 margin=6, nt=nt, nhills=2)
        lam, mu, rho = inputs._homog(p.ni, p.nj, p.nk)   # the driver's uniform medium
        p.lam, p.mu, p.rho = lam, mu, rho
    elif case == "sponge":
        p = dataclasses.replace(inputs.small_planar(nt=nt, pml=0), ablexp_layers=((6, 6), (6, 6), (6, 0)),
                                ablexp_ref_vel=((6000.0, 6000.0),) * 3)
    else:
        p = inputs.small_planar(nt=nt)
    par = par_files.write_case(p, str(tmp_path / "case"), nt=nt, io_time_skip=skip, medium=medium)
    r = subprocess.run([_driver(), par], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = json.load(open(par))["output_dir"]
    ds = [par_files.read_fault_output(os.path.join(out, f"fault_i{x}_px0_py0_pz0.nc")) for x in p.fault_x_index]
    # the reference's loop takes nt + 1 steps and writes a record before
    # every io_time_skip-th of them (drv_rk_curv_col.cu:209-227)
    nt_total = nt + 1
    nrec = (nt_total + skip - 1) // skip
    for d in ds:
        assert d["Tn"].shape == (nrec, p.nk, p.nj)
    p.max_records = nt_total
    s = Solver(p)
    for rec in range(nrec):
        for fi, d in enumerate(ds):
            np.testing.assert_allclose(d["time"][rec], rec * skip * p.dt, rtol=1e-6)
            for q, f in enumerate(par_files.FAULT_CMP):
                assert np.array_equal(d[f][rec], s.fault(f, fi)), (rec, fi, f)
        s.run(min(skip, nt_total - rec * skip))
    for fi, d in enumerate(ds):
        assert np.array_equal(d["Peak_vs"], s.fault("Peak_vs", fi))
        assert np.array_equal(d["Init_t0"], s.fault("Init_t0", fi))
        assert int(np.ravel(d["_attrs"]["i_index_with_ghosts_in_this_thread"])[0]) == p.fault_x_index[fi] + 2
    assert s.fault("Vs").max() > 0.05
    seis = s.stations()
    for q in range(len(p.stations)):
        for c, name in enumerate(par_files.CMP):
            fh, ih, kh, tr = par_files.read_sac(os.path.join(out, f"s{q}.{name}.sac"))
            assert ih[9] == nt_total and np.array_equal(tr, seis[q, c]), (q, name)
        # strain from the stress traces (the reference's conversion)
        i, j, k = [int(v) for v in p.stations[q]]
        lam, mu = float(p.lam[k, j, i]), float(p.mu[k, j, i])
        E2 = -lam / (2 * mu * (3 * lam + 2 * mu))
        _, _, _, exy = par_files.read_sac(os.path.join(out, f"s{q}.Exy.sac"))
        np.testing.assert_allclose(exy, 0.5 / mu * seis[q, 8], rtol=1e-5, atol=1e-30)
        _, _, _, exx = par_files.read_sac(os.path.join(out, f"s{q}.Exx.sac"))
        E1 = (lam + mu) / (mu * (3 * lam + 2 * mu))
        want = E2 * seis[q, 3:6].sum(0) - (E2 - E1) * seis[q, 3]
        np.testing.assert_allclose(exx, want, rtol=1e-4, atol=1e-3 * np.abs(want).max() + 1e-30)
    fseis = s.fault_stations()
    for q in range(len(p.fault_stations)):
        for c, name in enumerate(par_files.FAULT_CMP):
            _, _, _, tr = par_files.read_sac(os.path.join(out, f"fault_f{q}.{name}.sac"))
            assert np.array_equal(tr, fseis[q, c]), (q, name)
    # peak surface motion: the library's values in the interior of the
    # ghost-inclusive plane, zeros in the ghosts
    if not p.free_surface:
        assert not os.path.exists(os.path.join(out, "PG_V_A_D_px0_py0_pz0.nc"))
        return
    pg = par_files.read_surface_peaks(os.path.join(out, "PG_V_A_D_px0_py0_pz0.nc"))
    mine = s.surface_peaks()
    for c, name in enumerate(PEAK_FIELDS):
        v = pg[name]
        assert v.shape == (p.nj + 6, p.ni + 6)
        assert np.array_equal(v[3:-3, 3:-3], mine[c]), name
        assert not v[:3].any() and not v[:, :3].any()
    assert mine[0].max() > 0
    assert list(np.ravel(pg["_attrs"]["count_index_of_physical_points"])) == [p.ni, p.nj]


def test_case_writer_boundary_blocks(tmp_path):
    """par.json of a sponge case: "ablexp" {number_of_layers, ref_vel} on the
    five absorbing faces and "free" on the top, as par_t.cu:160-312 reads them."""
    p = dataclasses.replace(inputs.small_planar(nt=4, pml=0), ablexp_layers=((6, 6), (5, 5), (4, 0)),
                            ablexp_ref_vel=((6000.0, 5900.0), (5800.0, 5700.0), (5600.0, 5500.0)))
    par = json.load(open(par_files.write_case(p, str(tmp_path / "case"), nt=4)))
    names = [("boundary_x_left", 0, 0), ("boundary_x_right", 0, 1), ("boundary_y_front", 1, 0),
             ("boundary_y_back", 1, 1), ("boundary_z_bottom", 2, 0)]
    for key, d, s in names:
        blk = par[key]["ablexp"]
        assert blk["number_of_layers"] == p.ablexp_layers[d][s]
        assert blk["ref_vel"] == p.ablexp_ref_vel[d][s]
        assert "cfspml" not in par[key]
    assert "free" in par["boundary_z_top"]


def _template_par_text(case_dir, out_dir, p):
    """A par file laid out like the reference's shipped template
    (example/tpv/dynamic-cfspml.sh:53-205): its key set, its '#'-commented
    keys (some given twice, as the template does), its misspelt
    "check_nan_every_nummber_of_steps", the "check_stability" key that the
    reference's reader does not know, and export / line / slice / snapshot
    blocks; values for the small planar case.  Written as text because JSON
    objects with repeated keys have no Python dict form."""
    pml = ('{ "cfspml" : { "number_of_layers" : %d, "alpha_max" : 3.14, "beta_max" : 2.0, '
           '"ref_vel" : 6000.0 } }' % p.pml_layers[0][0])
    g = p.fault_grid[0]
    return f"""{{
  "number_of_total_grid_points_x" : {p.ni},
  "number_of_total_grid_points_y" : {p.nj},
  "number_of_total_grid_points_z" : {p.nk},
  "number_of_mpiprocs_y" : 1,
  "number_of_mpiprocs_z" : 1,
  "size_of_time_step" : {p.dt},
  "number_of_time_steps" : 4,
  "#time_window_length" : 10,
  "check_stability" : 1,
  "io_time_skip" : 1,
  "dynamic_method" : {p.dynamic_method},
  "fault_grid" : [{g[0]}, {g[1]}, {g[2]}, {g[3]}],
  "fault_x_index" : [ {p.fault_x_index[0]} ],
  "welded_margin" : {p.welded_margin},
  "grid_generation_method" : {{
      "fault_plane" : {{
        "fault_geometry_dir" : "{case_dir}/fault_coord",
        "fault_init_stress_dir" : "{case_dir}/init_stress",
        "fault_inteval" : {p.fault_interval}
      }},
      "#grid_import" : {{ "import_dir" : "{case_dir}", "fault_init_stress_dir" : "{case_dir}" }}
  }},
  "is_export_grid" : 1,
  "grid_export_dir"   : "{out_dir}",
  "boundary_x_left" : {pml},
  "boundary_x_right" : {pml},
  "boundary_y_front" : {pml},
  "boundary_y_back" : {pml},
  "boundary_z_bottom" : {pml},
  "boundary_z_top" : {{ "free" : "timg" }},
  "metric_calculation_method" : {{ "#import" : "{out_dir}", "calculate" : 1 }},
  "is_export_metric" : 1,
  "medium" : {{
      "type" : "elastic_iso",
      "#input_way" : "infile_layer",
      "#input_way" : "binfile",
      "input_way" : "code",
      "#binfile" : {{ "size" : [11, 14, 12], "spacing" : [-10, 10, 10], "origin" : [0.0, 0.0, 0.0],
                     "dim1" : "z", "dim2" : "x", "dim3" : "y" }},
      "#import" : "{out_dir}",
      "code" : "",
      "#equivalent_medium_method" : "loc",
      "#equivalent_medium_method" : "har"
  }},
  "is_export_media" : 1,
  "media_export_dir"  : "{out_dir}",
  "#visco_config" : {{ "type" : "graves_Qs", "Qs_freq" : 1.0 }},
  "output_dir" : "{out_dir}",
  "in_station_file" : "{case_dir}/stations.txt",
  "fault_station_file" : "{case_dir}/fault_stations.txt",
  "#receiver_line" : [ {{ "name" : "line_x_1", "grid_index_start" : [ 1, 9, 9 ],
                         "grid_index_incre" : [ 1, 0, 0 ], "grid_index_count" : 5 }} ],
  "#slice" : {{ "x_index" : [ 11 ], "y_index" : [ 12 ], "z_index" : [ 13 ] }},
  "#snapshot" : [ {{ "name" : "volume_vel", "grid_index_start" : [ 1, 1, {p.nk} ],
                    "grid_index_count" : [ {p.ni}, {p.nj}, 1 ], "grid_index_incre" : [ 1, 1, 1 ],
                    "time_index_start" : 0, "time_index_incre" : 1, "save_velocity" : 1,
                    "save_stress" : 0, "save_strain" : 0 }} ],
  "check_nan_every_nummber_of_steps" : 0,
  "output_all" : 0
}}
"""


def test_driver_accepts_the_reference_par_template(cgfd_lib, tmp_path):
    """cgfd_run --check (inputs and host set-up, no GPU) on a par file laid
    out like the reference's own template: every key is either used or
    reported as ignored, and the run is configured as the reference would
    configure it (the uniform medium of input_way "code", 4 + 1 steps)."""
    from cgfd import Problem  # noqa: F401
    lam, mu, rho = inputs._homog(36, 56, 32)
    p = inputs.small_planar(nt=4)
    p.lam, p.mu, p.rho = lam, mu, rho
    case = str(tmp_path / "case")
    par_files.write_case(p, case, nt=4, medium="code")
    fs = os.path.join(case, "fault_stations.txt")
    if not os.path.exists(fs):
        with open(fs, "w") as fh:
            fh.write("1\nf0 1 28.0 22.0\n")
    out = str(tmp_path / "out")
    os.makedirs(out)
    par = tmp_path / "template.json"
    par.write_text(_template_par_text(case, out, p))
    exe = os.path.join(ROOT, "gpu-cgfd3d-dynamic_b200", "lib", "cgfd_run")
    r = subprocess.run([exe, "--check", str(par)], capture_output=True, text=True, timeout=120,
                       env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert r.returncode == 0, r.stderr
    err = r.stderr
    for k in ("#time_window_length", "#visco_config", "#receiver_line", "#slice", "#snapshot"):
        assert f"{k}: commented out, ignored" in err, k
    for k in ("check_stability", "check_nan_every_nummber_of_steps"):
        assert f"{k}: not a key of the reference's par file, ignored" in err, k
    for k in ("is_export_grid", "grid_export_dir", "is_export_metric", "is_export_media", "media_export_dir",
              "output_all"):
        assert f"{k}: output not produced by this driver, ignored" in err, k
    for k in ("number_of_mpiprocs_y", "number_of_mpiprocs_z"):
        assert f"{k}: no effect on a single-GPU run, ignored" in err, k
    for k in ("number_of_total_grid_points_x", "medium", "metric_calculation_method", "boundary_z_top"):
        assert f"{k}:" not in err, k
    want = (f"grid {p.ni} x {p.nj} x {p.nk}, dt {p.dt:g}", "5 steps", "1 fault(s), dynamic_method 2",
            "free surface 1", f"{len(p.stations)} station(s)")
    for w in want:
        assert w in r.stdout, (w, r.stdout)


def test_reference_case_writer_keys(tmp_path):
    """The par file the reference-pin tests give the reference's own solver
    (tests/refcase.py) sets every top-level key its reader leaves
    uninitialised otherwise (par_t.cu:64-900: slices, snapshots, receiver
    lines, exports, the NaN check), keeps the welded margin at the
    reference's fixed 40, and is accepted as it is by cgfd_run --check."""
    import refcase
    p = inputs.tpv_planar(ni=40, nj=100, nk=60, nt=3, pml=5, nsta=3)
    par = refcase.write_reference_case(p, str(tmp_path / "case"), nt=3, medium="code")
    d = json.load(open(par))
    for k in ("receiver_line", "slice", "snapshot", "is_export_grid", "is_export_metric", "is_export_media",
              "grid_export_dir", "media_export_dir", "check_nan_every_number_of_steps", "output_all",
              "in_station_file", "fault_station_file", "metric_calculation_method"):
        assert k in d, k
    assert "welded_margin" not in d
    assert d["slice"] == {"x_index": [], "y_index": [], "z_index": []}
    with pytest.raises(ValueError):
        refcase.write_reference_case(inputs.small_planar(nt=3), str(tmp_path / "c2"), nt=3)   # margin 10
    exe = os.path.join(ROOT, "gpu-cgfd3d-dynamic_b200", "lib", "cgfd_run")
    r = subprocess.run([exe, "--check", par], capture_output=True, text=True, timeout=120,
                       env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert r.returncode == 0, r.stderr
    assert "4 steps" in r.stdout
