"""Build the CPU oracle (test infrastructure) into oracle/_build/.

liboracle.so   -- float, the reference's arithmetic
liboracle64.so -- double, for error estimates of the float paths
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")


def build(verbose=False):
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(HERE, "oracle.cpp")
    outs = []
    for name, defs in (("liboracle.so", []), ("liboracle64.so", ["-DORACLE_DOUBLE"])):
        dst = os.path.join(OUT, name)
        if os.path.exists(dst) and os.path.getmtime(dst) > max(
                os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "oracle.h")),
                os.path.getmtime(os.path.join(HERE, "..", "include", "cgfd.h"))):
            outs.append(dst)
            continue
        # -ffp-contract=off keeps each multiply and add separately rounded,
        # as the reference's expressions are written
        cmd = ["g++", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
               "-Wall", "-Wno-unused-variable", "-Wno-unused-but-set-variable"] + defs + [src, "-o", dst]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        outs.append(dst)
    return outs


if __name__ == "__main__":
    print(build(verbose=True))
    sys.exit(0)
