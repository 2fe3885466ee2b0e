"""Build libcgfd.so (sm_100a) in-tree: gpu-cgfd3d-dynamic_b200/lib/libcgfd.so,
and libcgfd64.so, the same kernels computing in double.

nvcc cross-compiles for sm_100a without a GPU; the host set-up is g++ with
OpenMP.  Objects go to gpu-cgfd3d-dynamic_b200/_build/.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libcgfd.so")
# the same kernels computing in double (-DCGFD_FP64), for error statements
# of the float build against a double build on the same inputs
LIB64 = os.path.join(LIBDIR, "libcgfd64.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"

# (source, object, extra flags): the volume kernels build as one unit per
# kernel kind so that they compile in parallel
CU = [("volume.cu", f"volume_k{k}.cu.o", [f"-DCGFD_VOLUME_KIND={k}"]) for k in range(8)] + [
    (f, f + ".o", []) for f in ("fault.cu", "boundary.cu", "noalloc.cu", "api.cu")]
CPP = ["setup.cpp"]
DRIVER = os.path.join(HERE, "driver")
DRIVER_SRC = ["cgfd_run.cpp", "ncclassic.cpp", "sac.cpp"]
DRIVER_BIN = os.path.join(HERE, "lib", "cgfd_run")
HEADERS = ["common.h", "ops.cuh", "setup.h", "real.h"]


def _newer(dst, srcs):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "cgfd.h")]
    objs = []
    for f in CPP:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        if _newer(obj, [src] + hdrs):
            cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        objs.append(obj)
    jobs = []
    objs64 = list(objs)
    for variant, defs, dst in (("", [], objs), ("64", ["-DCGFD_FP64"], objs64)):
        for f, o, extra in CU:
            src, obj = os.path.join(CSRC, f), os.path.join(BUILD, o.replace(".o", variant + ".o"))
            if _newer(obj, [src] + hdrs) or (ptxas_info and not variant):
                cmd = [NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                       "--expt-relaxed-constexpr"] + defs + extra + ["-c", src, "-o", obj]
                if ptxas_info and not variant:
                    cmd += ["-Xptxas", "-v"]
                jobs.append(cmd)
            dst.append(obj)
    if jobs:
        from concurrent.futures import ThreadPoolExecutor
        if verbose:
            for cmd in jobs:
                print(" ".join(cmd))
        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
            results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs))
        for cmd, r in zip(jobs, results):
            if r.stdout or r.stderr:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, cmd)
    for lib, ob in ((LIB, objs), (LIB64, objs64)):
        if _newer(lib, ob):
            cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + ob + ["-lgomp"]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    # the par-file driver, linked against the library with an rpath to it
    dsrc = [os.path.join(DRIVER, f) for f in DRIVER_SRC]
    dhdr = [os.path.join(DRIVER, f) for f in ("json.h", "ncclassic.h", "sac.h")] + hdrs
    if _newer(DRIVER_BIN, dsrc + dhdr + [LIB]):
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-pthread", "-o", DRIVER_BIN] + dsrc + \
              ["-L", LIBDIR, "-lcgfd", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
