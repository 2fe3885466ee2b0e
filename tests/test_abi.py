"""CPU checks of the C-ABI boundary: the sm_100a library builds, loads, exports
every entry point include/cgfd.h declares, and its config struct has the
same layout in C and in the Python binding."""
import ctypes as C
import os
import re
import subprocess

import pytest

import cgfd
from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "cgfd.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cgfd_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("cgfd_create", "cgfd_run", "cgfd_get_fault", "cgfd_get_stations", "cgfd_destroy",
              "cgfd_last_error", "cgfd_checkpoint", "cgfd_restore"):
        assert n in names


def test_library_exports_all(cgfd_lib):
    missing = [n for n in declared_functions() if not hasattr(cgfd_lib, n)]
    assert not missing, missing
    assert cgfd_lib.cgfd_abi_version() == 2


def test_config_default(cgfd_lib):
    c = cgfd.CgfdConfig()
    cgfd_lib.cgfd_config_default(C.byref(c))
    assert c.welded_margin == 40 and c.dynamic_method == 2 and c.check_stability == 1
    assert abs(c.pml_alpha_max[0][0] - 3.14) < 1e-6


def test_config_layout_matches_c(tmp_path):
    fields = [f[0] for f in cgfd.CgfdConfig._fields_]
    cname = {"lam": "lambda"}
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){",
           'printf("%zu\\n", sizeof(cgfd_config));']
    for f in fields:
        src.append(f'printf("%zu\\n", offsetof(cgfd_config, {cname.get(f, f)}));')
    src.append("return 0;}")
    (tmp_path / "l.c").write_text("\n".join(src))
    subprocess.check_call(["gcc", str(tmp_path / "l.c"), "-o", str(tmp_path / "l")])
    out = [int(x) for x in subprocess.check_output([str(tmp_path / "l")]).split()]
    assert out[0] == C.sizeof(cgfd.CgfdConfig)
    for f, off in zip(fields, out[1:]):
        assert getattr(cgfd.CgfdConfig, f).offset == off, f


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_loudly(cgfd_lib):
    import inputs
    p = inputs.small_planar(nt=2)
    with pytest.raises(cgfd.CgfdError, match="ERR_NODEVICE"):
        cgfd.Solver(p)


def test_invalid_config_rejected_before_device(cgfd_lib):
    c = cgfd.CgfdConfig()
    cgfd_lib.cgfd_config_default(C.byref(c))
    h = C.c_void_p()
    rc = cgfd_lib.cgfd_create(C.byref(c), C.byref(h))
    assert rc in (-1, -6)      # ERR_ARG, or ERR_NODEVICE when no GPU is present
    assert cgfd_lib.cgfd_last_error()


def _bad_cases():
    import dataclasses
    import numpy as np
    import inputs
    p = inputs.small_planar(nt=2)
    rep = dataclasses.replace
    rho0 = p.rho.copy()
    rho0[3, 4, 5] = 0.0
    dc0 = p.Dc.copy()
    dc0[0, 10, 20] = 0.0
    return [
        ("grid too small", rep(p, ni=8, nj=8, nk=8), "at least 12"),
        ("dynamic method", rep(p, dynamic_method=3), "dynamic_method"),
        ("dt not positive", rep(p, dt=0.0), "dt must be positive"),
        ("pml too wide", rep(p, pml_layers=((30, 5), (5, 5), (5, 0))), "pml_layers out of range"),
        ("sponge with pml", rep(p, ablexp_layers=((4, 4), (0, 0), (0, 0))), "cannot be combined"),
        ("sponge on free top", rep(p, pml_layers=((0, 0), (0, 0), (0, 0)), ablexp_layers=((0, 0), (0, 0), (0, 4))),
         "free top"),
        ("station outside", rep(p, stations=np.array([[p.ni + 2, 3, 3]], np.float32)), "station outside"),
        ("fault station outside", rep(p, fault_stations=np.array([[p.nj + 5, 2]], np.float32)), "fault station"),
        ("fault near the x side", rep(p, fault_x_index=[3]), "fault_x_index"),
        ("medium", rep(p, rho=rho0), "medium must have"),
        ("Dc", rep(p, Dc=dc0), "Dc must be positive"),
        ("dt above the CFL limit", rep(p, dt=0.05), "CFL"),
    ]


@pytest.mark.parametrize("case", range(12))
def test_prepare_rejects_invalid_input(cgfd_lib, case):
    """cgfd_prepare (host only) rejects each invalid input with a status code and
    a message naming the problem, where the reference aborts, exits or runs on."""
    name, prob, msg = _bad_cases()[case]
    with pytest.raises(cgfd.CgfdError, match=msg):
        cgfd.Setup(prob)


def test_prepare_valid_inputs(cgfd_lib):
    """The same host set-up accepts the valid variants: the sponge in place of the
    PML, and a dt above the CFL limit when the check is switched off."""
    import dataclasses
    import inputs
    p = inputs.small_planar(nt=2)
    s = cgfd.Setup(p)
    assert 0.01 < s.dt_max() < 0.05 and s.upload_bytes > 0
    s.close()
    sp = dataclasses.replace(p, pml_layers=((0, 0), (0, 0), (0, 0)), ablexp_layers=((5, 5), (5, 5), (5, 0)))
    cgfd.Setup(sp).close()
    cgfd.Setup(dataclasses.replace(p, dt=0.05, check_stability=0)).close()
