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
    for d in ds:
        assert d["Tn"].shape == (nt // skip, p.nk, p.nj)
    s = Solver(p)
    for rec in range(nt // skip):
        for fi, d in enumerate(ds):
            np.testing.assert_allclose(d["time"][rec], rec * skip * p.dt, rtol=1e-6)
            for q, f in enumerate(par_files.FAULT_CMP):
                assert np.array_equal(d[f][rec], s.fault(f, fi)), (rec, fi, f)
        s.run(skip)
    for fi, d in enumerate(ds):
        assert np.array_equal(d["Peak_vs"], s.fault("Peak_vs", fi))
        assert np.array_equal(d["Init_t0"], s.fault("Init_t0", fi))
        assert int(np.ravel(d["_attrs"]["i_index_with_ghosts_in_this_thread"])[0]) == p.fault_x_index[fi] + 2
    assert s.fault("Vs").max() > 0.05
    seis = s.stations()
    for q in range(len(p.stations)):
        for c, name in enumerate(par_files.CMP):
            fh, ih, kh, tr = par_files.read_sac(os.path.join(out, f"s{q}.{name}.sac"))
            assert ih[9] == nt and np.array_equal(tr, seis[q, c]), (q, name)
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
