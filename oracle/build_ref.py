"""Build the reference's own forward solver, unmodified, into oracle/_ref/.

Test infrastructure.  hpc-lee/gpu-CGFD3D-dynamic builds ``main`` from
src/forward/*.cu and src/lib/*.cu (nvcc, relocatable device code) and
src/media/*.cpp (mpicxx), linked against MPI and netCDF (its Makefile).  This
recipe compiles the same source files where they lie in the reference tree,
for sm_100a, against the single-rank MPI and netCDF-classic stand-ins in
oracle/refshim/ instead of those libraries, and links
oracle/_ref/cgfd_ref_main.  Run it as ``cgfd_ref_main par.json 0`` on a
machine with a GPU; it writes the reference's fault netCDF and SAC files.

The reference tree is read from $CGFD_REFERENCE (default /root/reference);
nothing is written there.  The built program is never linked into, loaded
by or called from the solver library: only tests compare its outputs with
the oracle's and the solver's.
"""
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
EXE = os.path.join(OUT, "cgfd_ref_main")
SHIM = os.path.join(HERE, "refshim")
NCDIR = os.path.join(HERE, "..", "gpu-cgfd3d-dynamic_b200", "driver")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = "sm_100a"


def reference_root():
    return os.environ.get("CGFD_REFERENCE", "/root/reference")


def sources(root):
    fwd = sorted(glob.glob(os.path.join(root, "src", "forward", "*.cu")))
    lib = sorted(glob.glob(os.path.join(root, "src", "lib", "*.cu")))
    med = sorted(glob.glob(os.path.join(root, "src", "media", "*.cpp")))
    return fwd + lib, med


def available():
    """True when the reference tree is present (it is not on GPU boxes,
    which use the program built here)."""
    fwd, _ = sources(reference_root())
    return len(fwd) > 0


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    return cmd, r


def build(verbose=False, jobs=None):
    root = reference_root()
    cu, cpp = sources(root)
    if not cu:
        if os.path.exists(EXE):
            return EXE
        raise FileNotFoundError(f"reference sources not found under {root}")
    os.makedirs(OBJ, exist_ok=True)
    inc = ["-I", SHIM, "-I", os.path.join(root, "src", "lib"), "-I", os.path.join(root, "src", "media"),
           "-I", os.path.join(root, "src", "forward")]
    shim_src = [os.path.join(SHIM, "refshim.cpp"), os.path.join(NCDIR, "ncclassic.cpp")]
    shim_hdr = [os.path.join(SHIM, "mpi.h"), os.path.join(SHIM, "netcdf.h"), os.path.join(NCDIR, "ncclassic.h")]
    hdr_t = max(os.path.getmtime(h) for h in shim_hdr)
    cmds, objs = [], []
    # the reference's own flags (Makefile: -O3 -std=c++11 -w -rdc=true), arch sm_100a
    for s in cu:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t):
            cmds.append([NVCC, "-O3", f"-arch={ARCH}", "-std=c++11", "-w", "-rdc=true"] + inc + ["-c", s, "-o", o])
    for s in cpp:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t):
            cmds.append(["g++", "-O3", "-std=c++11", "-w"] + inc + ["-c", s, "-o", o])
    for s in shim_src:
        o = os.path.join(OBJ, "shim_" + os.path.basename(s) + ".o")
        objs.append(o)
        if not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t):
            cmds.append(["g++", "-O2", "-std=c++17", "-Wall", "-I", SHIM, "-I", NCDIR, "-c", s, "-o", o])
    if cmds:
        with ThreadPoolExecutor(max_workers=jobs or max(1, os.cpu_count() or 1)) as ex:
            for cmd, r in ex.map(_run, cmds):
                if verbose:
                    print(" ".join(cmd))
                if r.returncode != 0:
                    sys.stderr.write(r.stdout + r.stderr)
                    raise subprocess.CalledProcessError(r.returncode, cmd)
    if not os.path.exists(EXE) or os.path.getmtime(EXE) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, f"-arch={ARCH}", "-o", EXE] + objs + ["-lm"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return EXE


if __name__ == "__main__":
    print(build(verbose=True))
