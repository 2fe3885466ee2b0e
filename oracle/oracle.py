"""ctypes binding of the CPU oracle (test infrastructure only).

Loaded by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline and
reference arm, as the checker.  Mirrors the product's Solver API so parity
tests read the same on both sides.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "gpu-cgfd3d-dynamic_b200"))
from cgfd import CgfdConfig, FAULT_FIELDS, WAVE_COMPONENTS, Problem  # noqa: E402

_libs = {}
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def load(double=False):
    name = "liboracle64.so" if double else "liboracle.so"
    if name in _libs:
        return _libs[name]
    path = os.path.join(HERE, "_build", name)
    if not os.path.exists(path):
        from build_oracle import build  # type: ignore
        build()
    lib = C.CDLL(path)
    vp = C.c_void_p
    lib.oracle_create.argtypes = [C.POINTER(CgfdConfig), C.POINTER(vp)]
    lib.oracle_run.argtypes = [vp, C.c_int]
    lib.oracle_get_fault.argtypes = [vp, C.c_int, C.c_int, _fp]
    lib.oracle_get_stations.argtypes = [vp, _fp, _ip]
    lib.oracle_get_fault_stations.argtypes = [vp, _fp, _ip]
    lib.oracle_get_wavefield.argtypes = [vp, C.c_int, _fp]
    lib.oracle_set_wavefield.argtypes = [vp, C.c_int, _fp]
    lib.oracle_get_metric.argtypes = [vp, C.c_int, _fp]
    lib.oracle_dt_max.argtypes = [vp, _fp]
    lib.oracle_get_surface_peaks.argtypes = [vp, _fp]
    lib.oracle_set_threads.argtypes = [C.c_int]
    lib.oracle_destroy.argtypes = [vp]
    lib.oracle_destroy.restype = None
    lib.oracle_last_error.restype = C.c_char_p
    _libs[name] = lib
    return lib


sys.path.insert(0, HERE)


class OracleSolver:
    def __init__(self, prob: Problem, double=False, threads=0):
        self.lib = load(double)
        if threads:
            self.lib.oracle_set_threads(int(threads))
        self.prob = prob
        self._cfg = prob.to_config()
        h = C.c_void_p()
        rc = self.lib.oracle_create(C.byref(self._cfg), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"oracle_create failed ({rc}): {self.lib.oracle_last_error().decode()}")
        self.h = h

    def run(self, n):
        rc = self.lib.oracle_run(self.h, int(n))
        if rc != 0:
            raise RuntimeError(self.lib.oracle_last_error().decode())

    def fault(self, field, fault_id=0):
        if isinstance(field, str):
            field = FAULT_FIELDS.index(field)
        p = self.prob
        out = np.empty((p.nk, p.nj), np.float32)
        self.lib.oracle_get_fault(self.h, fault_id, field, out.ctypes.data_as(_fp))
        return out

    def stations(self):
        n = C.c_int()
        self.lib.oracle_get_stations(self.h, None, C.byref(n))
        ns = 0 if self.prob.stations is None else len(self.prob.stations)
        out = np.empty((ns, 9, n.value), np.float32)
        self.lib.oracle_get_stations(self.h, out.ctypes.data_as(_fp), C.byref(n))
        return out

    def fault_stations(self):
        n = C.c_int()
        self.lib.oracle_get_fault_stations(self.h, None, C.byref(n))
        ns = 0 if self.prob.fault_stations is None else len(self.prob.fault_stations)
        out = np.empty((ns, 9, n.value), np.float32)
        self.lib.oracle_get_fault_stations(self.h, out.ctypes.data_as(_fp), C.byref(n))
        return out

    def surface_peaks(self):
        p = self.prob
        out = np.empty((15, p.nj, p.ni), np.float32)
        rc = self.lib.oracle_get_surface_peaks(self.h, out.ctypes.data_as(_fp))
        if rc != 0:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        return out

    def wavefield(self, cmp):
        if isinstance(cmp, str):
            cmp = WAVE_COMPONENTS.index(cmp)
        p = self.prob
        out = np.empty((p.nk, p.nj, p.ni), np.float32)
        self.lib.oracle_get_wavefield(self.h, cmp, out.ctypes.data_as(_fp))
        return out

    def set_wavefield(self, cmp, arr):
        if isinstance(cmp, str):
            cmp = WAVE_COMPONENTS.index(cmp)
        a = np.ascontiguousarray(arr, np.float32)
        self.lib.oracle_set_wavefield(self.h, cmp, a.ctypes.data_as(_fp))

    def metric(self, cmp):
        p = self.prob
        out = np.empty((p.nk, p.nj, p.ni), np.float32)
        self.lib.oracle_get_metric(self.h, cmp, out.ctypes.data_as(_fp))
        return out

    def dt_max(self):
        v = C.c_float()
        self.lib.oracle_dt_max(self.h, C.byref(v))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
