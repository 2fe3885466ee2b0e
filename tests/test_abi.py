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
