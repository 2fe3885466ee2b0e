"""Host-side Python mirror of the solver's C ABI (include/cgfd.h).

The reference drives its forward path from ``main par.json``
(src/forward/main_curv_col_el_3d.cu:45-749): set-up on the host, then
``drv_rk_curv_col_allstep`` (src/forward/drv_rk_curv_col.cu:29-52) runs the
time loop on the GPU.  Here a :class:`Problem` holds the same inputs as
numpy arrays (grid or fault surfaces, medium, fault initial stress and
friction, stations) and :class:`Solver` drives ``libcgfd.so`` through ctypes.

``Solver`` raises if the CUDA library is missing or no GPU is present: there
is no CPU fallback in the product.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CGFD_LIB", os.path.join(HERE, "lib", "libcgfd.so"))
# the same kernels computing in double, for error statements of the float build
LIB64_PATH = os.path.join(HERE, "lib", "libcgfd64.so")

MAX_FAULTS = 8
GRID_FAULT_PLANE = 0
GRID_IMPORT = 1

FAULT_FIELDS = ["Tn", "Ts1", "Ts2", "Vs", "Vs1", "Vs2", "Slip", "Slip1", "Slip2",
                "Peak_vs", "Init_t0"]
WAVE_COMPONENTS = ["Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Tyz", "Txz", "Txy"]
# surface peak fields of cgfd_get_surface_peaks (the PG_V_A_D file's variables)
PEAK_FIELDS = ["PGV", "PGVh", "PGVx", "PGVy", "PGVz", "PGA", "PGAh", "PGAx", "PGAy", "PGAz",
               "PGD", "PGDh", "PGDx", "PGDy", "PGDz"]

ERRORS = {0: "OK", -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_NOMEM", -4: "ERR_UNSTABLE",
          -5: "ERR_DT", -6: "ERR_NODEVICE", -7: "ERR_STATE"}

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class CgfdConfig(C.Structure):
    """ctypes image of ``cgfd_config`` (include/cgfd.h)."""
    _fields_ = [
        ("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int),
        ("dt", C.c_float),
        ("check_stability", C.c_int),
        ("dynamic_method", C.c_int),
        ("num_faults", C.c_int),
        ("fault_x_index", C.c_int * MAX_FAULTS),
        ("fault_grid", (C.c_int * 4) * MAX_FAULTS),
        ("welded_margin", C.c_int),
        ("free_surface", C.c_int),
        ("pml_layers", (C.c_int * 2) * 3),
        ("pml_alpha_max", (C.c_float * 2) * 3),
        ("pml_beta_max", (C.c_float * 2) * 3),
        ("pml_ref_vel", (C.c_float * 2) * 3),
        ("grid_mode", C.c_int),
        ("fault_interval", C.c_float),
        ("fault_x", _fp), ("fault_y", _fp), ("fault_z", _fp),
        ("x3d", _fp), ("y3d", _fp), ("z3d", _fp),
        ("lam", _fp), ("mu", _fp), ("rho", _fp),
        ("T0x", _fp), ("T0y", _fp), ("T0z", _fp),
        ("mu_s", _fp), ("mu_d", _fp), ("Dc", _fp), ("C0", _fp),
        ("num_stations", C.c_int),
        ("station_ijk", _fp),
        ("num_fault_stations", C.c_int),
        ("fault_station_fault", _ip),
        ("fault_station_jk", _fp),
        ("max_records", C.c_int),
        ("ablexp_layers", (C.c_int * 2) * 3),
        ("ablexp_ref_vel", (C.c_float * 2) * 3),
    ]


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


@dataclass
class Problem:
    """Inputs of one forward run, reference axes (x normal, y strike, z up).

    3-D arrays are [nk, nj, ni]; fault-plane arrays are [num_faults, nk, nj].
    Index fields (fault_x_index, fault_grid) are 1-based as in the par file.
    """
    ni: int
    nj: int
    nk: int
    dt: float
    lam: np.ndarray
    mu: np.ndarray
    rho: np.ndarray
    fault_x_index: list
    fault_grid: list
    T0x: np.ndarray
    T0y: np.ndarray
    T0z: np.ndarray
    mu_s: np.ndarray
    mu_d: np.ndarray
    Dc: np.ndarray
    C0: np.ndarray
    dynamic_method: int = 2
    welded_margin: int = 40
    free_surface: int = 1
    pml_layers: tuple = ((0, 0), (0, 0), (0, 0))
    pml_alpha_max: tuple = ((3.14, 3.14), (3.14, 3.14), (3.14, 3.14))
    pml_beta_max: tuple = ((2.0, 2.0), (2.0, 2.0), (2.0, 2.0))
    pml_ref_vel: tuple = ((6000.0, 6000.0), (6000.0, 6000.0), (6000.0, 6000.0))
    ablexp_layers: tuple = ((0, 0), (0, 0), (0, 0))
    ablexp_ref_vel: tuple = ((6000.0, 6000.0), (6000.0, 6000.0), (6000.0, 6000.0))
    grid_mode: int = GRID_FAULT_PLANE
    fault_interval: float = 0.0
    fault_x: np.ndarray = None
    fault_y: np.ndarray = None
    fault_z: np.ndarray = None
    x3d: np.ndarray = None
    y3d: np.ndarray = None
    z3d: np.ndarray = None
    stations: np.ndarray = None          # [n, 3] 0-based (i, j, k)
    fault_stations: np.ndarray = None    # [n, 2] 0-based (j, k)
    fault_station_fault: np.ndarray = None
    max_records: int = 0
    check_stability: int = 1
    name: str = "problem"
    _keep: list = field(default_factory=list, repr=False)

    @property
    def num_faults(self):
        return len(self.fault_x_index)

    @property
    def points(self):
        return self.ni * self.nj * self.nk

    def to_config(self) -> CgfdConfig:
        """Build the C struct; the arrays stay alive as long as this Problem."""
        c = CgfdConfig()
        c.ni, c.nj, c.nk = self.ni, self.nj, self.nk
        c.dt = self.dt
        c.check_stability = int(self.check_stability)
        c.dynamic_method = int(self.dynamic_method)
        c.num_faults = self.num_faults
        for f in range(self.num_faults):
            c.fault_x_index[f] = int(self.fault_x_index[f])
            for q in range(4):
                c.fault_grid[f][q] = int(self.fault_grid[f][q])
        c.welded_margin = int(self.welded_margin)
        c.free_surface = int(self.free_surface)
        for d in range(3):
            for s in range(2):
                c.pml_layers[d][s] = int(self.pml_layers[d][s])
                c.pml_alpha_max[d][s] = float(self.pml_alpha_max[d][s])
                c.pml_beta_max[d][s] = float(self.pml_beta_max[d][s])
                c.pml_ref_vel[d][s] = float(self.pml_ref_vel[d][s])
                c.ablexp_layers[d][s] = int(self.ablexp_layers[d][s])
                c.ablexp_ref_vel[d][s] = float(self.ablexp_ref_vel[d][s])
        c.grid_mode = int(self.grid_mode)
        c.fault_interval = float(self.fault_interval)
        keep = []

        def ptr(a, ct=C.c_float):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float32 if ct is C.c_float else np.int32)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(ct))

        c.fault_x, c.fault_y, c.fault_z = ptr(self.fault_x), ptr(self.fault_y), ptr(self.fault_z)
        c.x3d, c.y3d, c.z3d = ptr(self.x3d), ptr(self.y3d), ptr(self.z3d)
        c.lam, c.mu, c.rho = ptr(self.lam), ptr(self.mu), ptr(self.rho)
        c.T0x, c.T0y, c.T0z = ptr(self.T0x), ptr(self.T0y), ptr(self.T0z)
        c.mu_s, c.mu_d, c.Dc, c.C0 = ptr(self.mu_s), ptr(self.mu_d), ptr(self.Dc), ptr(self.C0)
        st = self.stations
        c.num_stations = 0 if st is None else int(len(st))
        c.station_ijk = ptr(None if st is None else np.asarray(st, np.float32).reshape(-1, 3))
        fs = self.fault_stations
        c.num_fault_stations = 0 if fs is None else int(len(fs))
        if fs is not None:
            ff = self.fault_station_fault
            if ff is None:
                ff = np.zeros(len(fs), np.int32)
            c.fault_station_fault = ptr(np.asarray(ff, np.int32), C.c_int)
            c.fault_station_jk = ptr(np.asarray(fs, np.float32).reshape(-1, 2))
        c.max_records = int(self.max_records)
        self._keep = keep
        return c


class CgfdError(RuntimeError):
    pass


_libs = {}


def load_library(path: str = LIB_PATH):
    """Load libcgfd.so (or, given its path, libcgfd64.so); raises if it has
    not been built."""
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise CgfdError(f"libcgfd.so not built at {path}: run build.py (or __graft_entry__.build())")
    lib = C.CDLL(path)
    vp = C.c_void_p
    lib.cgfd_abi_version.restype = C.c_int
    lib.cgfd_config_default.argtypes = [C.POINTER(CgfdConfig)]
    lib.cgfd_create.argtypes = [C.POINTER(CgfdConfig), C.POINTER(vp)]
    lib.cgfd_run.argtypes = [vp, C.c_int]
    lib.cgfd_steps_done.argtypes = [vp, _ip]
    lib.cgfd_dt_max.argtypes = [vp, _fp]
    lib.cgfd_get_fault.argtypes = [vp, C.c_int, C.c_int, _fp]
    lib.cgfd_get_fault_all.argtypes = [vp, C.c_int, _fp]
    lib.cgfd_get_stations.argtypes = [vp, _fp, _ip]
    lib.cgfd_get_fault_stations.argtypes = [vp, _fp, _ip]
    lib.cgfd_get_wavefield.argtypes = [vp, C.c_int, _fp]
    lib.cgfd_get_surface_peaks.argtypes = [vp, _fp]
    lib.cgfd_release_cached_memory.argtypes = []
    lib.cgfd_set_wavefield.argtypes = [vp, C.c_int, _fp]
    lib.cgfd_checkpoint_size.argtypes = [vp, C.POINTER(C.c_ulonglong)]
    lib.cgfd_checkpoint.argtypes = [vp, vp, C.c_ulonglong]
    lib.cgfd_restore.argtypes = [vp, vp, C.c_ulonglong]
    lib.cgfd_last_launches.argtypes = [vp, C.POINTER(C.c_longlong)]
    lib.cgfd_destroy.argtypes = [vp]
    lib.cgfd_destroy.restype = None
    lib.cgfd_last_error.restype = C.c_char_p
    lib.cgfd_prepare.argtypes = [C.POINTER(CgfdConfig), C.POINTER(vp)]
    lib.cgfd_setup_bytes.argtypes = [vp, C.POINTER(C.c_ulonglong)]
    lib.cgfd_setup_dt_max.argtypes = [vp, _fp]
    lib.cgfd_upload.argtypes = [vp, C.POINTER(vp)]
    lib.cgfd_setup_free.argtypes = [vp]
    lib.cgfd_setup_free.restype = None
    lib.cgfd_set_timing.argtypes = [vp, C.c_int]
    lib.cgfd_last_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
    lib.cgfd_run_noalloc.argtypes = [vp, C.c_int]
    lib.cgfd_run_fault_output.argtypes = [vp, C.c_int, C.c_int, vp, C.c_longlong, _ip]
    lib.cgfd_ensemble_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(vp)]
    lib.cgfd_ensemble_run.argtypes = [vp, C.c_int]
    lib.cgfd_ensemble_destroy.argtypes = [vp]
    lib.cgfd_ensemble_destroy.restype = None
    lib.cgfd_last_kernel_timing.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                            C.POINTER(C.c_longlong)]
    _libs[path] = lib
    return lib


def load_library64():
    """libcgfd64.so: the solver's kernels built to compute and store in
    double, behind the same C ABI (float inputs widened, outputs narrowed)."""
    return load_library(LIB64_PATH)


def _fptr(a):
    return a.ctypes.data_as(_fp)


class Setup:
    """Host-side set-up of a problem (cgfd_prepare); needs no GPU."""

    def __init__(self, prob: Problem, lib=None):
        self.lib = lib or load_library()
        self.prob = prob
        self._cfg = prob.to_config()
        h = C.c_void_p()
        rc = self.lib.cgfd_prepare(C.byref(self._cfg), C.byref(h))
        if rc != 0:
            raise CgfdError(f"{ERRORS.get(rc, rc)}: {self.lib.cgfd_last_error().decode()}")
        self.h = h

    @property
    def upload_bytes(self):
        v = C.c_ulonglong()
        self.lib.cgfd_setup_bytes(self.h, C.byref(v))
        return v.value

    def dt_max(self):
        v = C.c_float()
        self.lib.cgfd_setup_dt_max(self.h, C.byref(v))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.cgfd_setup_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """A forward dynamic-rupture run on the current CUDA device."""

    def __init__(self, prob: Problem, lib=None, setup: Setup = None):
        self.lib = lib or load_library()
        self.prob = prob
        h = C.c_void_p()
        if setup is not None:
            self._check(self.lib.cgfd_upload(setup.h, C.byref(h)))
        else:
            self._cfg = prob.to_config()
            self._check(self.lib.cgfd_create(C.byref(self._cfg), C.byref(h)))
        self.h = h

    def set_timing(self, on=True):
        self._check(self.lib.cgfd_set_timing(self.h, int(bool(on))))

    def last_timing(self):
        """(run_ms, volume_ms, volume_launches) of the last run()."""
        a, b, n = C.c_double(), C.c_double(), C.c_longlong()
        self._check(self.lib.cgfd_last_timing(self.h, C.byref(a), C.byref(b), C.byref(n)))
        return a.value, b.value, n.value

    def run_noalloc(self, nsteps: int):
        """Advance like run(), allocating nothing (cgfd_run_noalloc): direct
        launches, traction scratch in the library's fixed device array.  Calls
        on one device must not overlap."""
        self._check(self.lib.cgfd_run_noalloc(self.h, int(nsteps)))

    def kernel_timing(self, which):
        """(ms, launches, points per launch) of the last run() with timing on:
        which 0 = the whole volume stage, 1 = the interior-box kernel."""
        a, n, p = C.c_double(), C.c_longlong(), C.c_longlong()
        self._check(self.lib.cgfd_last_kernel_timing(self.h, int(which), C.byref(a), C.byref(n), C.byref(p)))
        return a.value, n.value, p.value

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.cgfd_last_error().decode()
            raise CgfdError(f"{ERRORS.get(rc, rc)}: {msg}")

    def run(self, nsteps: int):
        self._check(self.lib.cgfd_run(self.h, int(nsteps)))

    def run_fault_output(self, nsteps: int, every: int = 1, out_ptr: int = None, max_records: int = None):
        """Advance nsteps steps, taking the fault fields before every step
        whose index is a multiple of `every` (cgfd_run_fault_output).  With
        out_ptr (e.g. a page-locked buffer's address) the records go there
        and their count is returned; otherwise a new array
        [records, faults, 11, nk, nj] is returned."""
        p = self.prob
        start = self.steps_done
        want = sum(1 for q in range(nsteps) if (start + q) % every == 0)
        n = C.c_int()
        if out_ptr is not None:
            cap = want if max_records is None else max_records
            self._check(self.lib.cgfd_run_fault_output(self.h, int(nsteps), int(every), C.c_void_p(out_ptr),
                                                       int(cap), C.byref(n)))
            return n.value
        out = np.empty((max(want, 1), p.num_faults, 11, p.nk, p.nj), np.float32)
        self._check(self.lib.cgfd_run_fault_output(self.h, int(nsteps), int(every), out.ctypes.data_as(C.c_void_p),
                                                   int(want), C.byref(n)))
        return out[:n.value]

    @property
    def steps_done(self):
        v = C.c_int()
        self._check(self.lib.cgfd_steps_done(self.h, C.byref(v)))
        return v.value

    def dt_max(self):
        v = C.c_float()
        self._check(self.lib.cgfd_dt_max(self.h, C.byref(v)))
        return v.value

    def fault(self, field, fault_id=0):
        if isinstance(field, str):
            field = FAULT_FIELDS.index(field)
        p = self.prob
        out = np.empty((p.nk, p.nj), np.float32)
        self._check(self.lib.cgfd_get_fault(self.h, fault_id, field, _fptr(out)))
        return out

    def fault_all(self, fault_id=0, out=None, out_ptr=None):
        """All 11 fault fields [11, nk, nj]; ``out_ptr`` (an address) lets the
        caller pass pinned host memory."""
        p = self.prob
        if out_ptr is not None:
            self._check(self.lib.cgfd_get_fault_all(self.h, fault_id, C.cast(out_ptr, _fp)))
            return None
        if out is None:
            out = np.empty((11, p.nk, p.nj), np.float32)
        self._check(self.lib.cgfd_get_fault_all(self.h, fault_id, _fptr(out)))
        return out

    def stations(self):
        n = C.c_int()
        self._check(self.lib.cgfd_get_stations(self.h, None, C.byref(n)))
        ns = 0 if self.prob.stations is None else len(self.prob.stations)
        out = np.empty((ns, 9, n.value), np.float32)
        self._check(self.lib.cgfd_get_stations(self.h, _fptr(out), C.byref(n)))
        return out

    def fault_stations(self):
        n = C.c_int()
        self._check(self.lib.cgfd_get_fault_stations(self.h, None, C.byref(n)))
        ns = 0 if self.prob.fault_stations is None else len(self.prob.fault_stations)
        out = np.empty((ns, 9, n.value), np.float32)
        self._check(self.lib.cgfd_get_fault_stations(self.h, _fptr(out), C.byref(n)))
        return out

    def surface_peaks(self):
        """Peak ground motion of the free surface, [15, nj, ni] in the order
        of ``PEAK_FIELDS``."""
        p = self.prob
        out = np.empty((15, p.nj, p.ni), np.float32)
        self._check(self.lib.cgfd_get_surface_peaks(self.h, _fptr(out)))
        return out

    def wavefield(self, cmp):
        if isinstance(cmp, str):
            cmp = WAVE_COMPONENTS.index(cmp)
        p = self.prob
        out = np.empty((p.nk, p.nj, p.ni), np.float32)
        self._check(self.lib.cgfd_get_wavefield(self.h, cmp, _fptr(out)))
        return out

    def set_wavefield(self, cmp, arr):
        if isinstance(cmp, str):
            cmp = WAVE_COMPONENTS.index(cmp)
        a = np.ascontiguousarray(arr, np.float32)
        self._check(self.lib.cgfd_set_wavefield(self.h, cmp, _fptr(a)))

    def checkpoint(self):
        n = C.c_ulonglong()
        self._check(self.lib.cgfd_checkpoint_size(self.h, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        self._check(self.lib.cgfd_checkpoint(self.h, buf.ctypes.data, n.value))
        return buf

    def restore(self, buf):
        self._check(self.lib.cgfd_restore(self.h, buf.ctypes.data, buf.nbytes))

    def last_launches(self):
        v = C.c_longlong()
        self._check(self.lib.cgfd_last_launches(self.h, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.cgfd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ensemble:
    """Independent solvers advanced together, one CUDA graph per step with a
    branch per member (cgfd_ensemble_*).  The members stay usable through
    their own getters; keep them alive while the ensemble exists."""

    def __init__(self, solvers):
        self.lib = load_library()
        self.members = list(solvers)
        arr = (C.c_void_p * len(self.members))(*[m.h for m in self.members])
        h = C.c_void_p()
        rc = self.lib.cgfd_ensemble_create(arr, len(self.members), C.byref(h))
        if rc != 0:
            raise CgfdError(f"{ERRORS.get(rc, rc)}: {self.lib.cgfd_last_error().decode()}")
        self.h = h

    def run(self, nsteps: int):
        rc = self.lib.cgfd_ensemble_run(self.h, int(nsteps))
        if rc != 0:
            raise CgfdError(f"{ERRORS.get(rc, rc)}: {self.lib.cgfd_last_error().decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.cgfd_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
