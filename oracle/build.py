"""Build recipe of the CPU oracle (test infrastructure only).

Compiles ``oracle/dfn_oracle.c`` with gcc into ``oracle/_build/libdfn_oracle.so``.
``-ffp-contract=off`` keeps FMA out of the restatement (the reference's
x86-64 -O1 Fortran build has none); OpenMP is used only to spread independent
receiver rows of the kernel sums over threads, so results do not depend on the
thread count.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libdfn_oracle.so")
SRC = os.path.join(HERE, "dfn_oracle.c")
HDR = os.path.join(os.path.dirname(HERE), "include", "dfn_b200.h")


def build(force=False):
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(SRC), os.path.getmtime(HDR))):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-std=c11", "-Wall",
           "-o", LIB + ".tmp", SRC, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("gcc failed:\n" + r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
