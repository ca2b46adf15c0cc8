"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/mrlbm_oracle.cpp into oracle/liborc.so with the reference's numerical
build conditions: baseline x86-64 (no FMA instructions), -ffp-contract=off, OpenMP for the
loops the reference parallelises (2d_mrlbm.f90:232, 407, 420, 430, 445).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "mrlbm_oracle.cpp")
OUT = os.path.join(HERE, "liborc.so")


def build(force: bool = False) -> str:
    if (not force and os.path.exists(OUT)
            and os.path.getmtime(OUT) >= os.path.getmtime(SRC)
            and os.path.getmtime(OUT) >= os.path.getmtime(os.path.join(HERE, "..", "include", "mrlbm.h"))):
        return OUT
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64", "-mtune=generic", "-ffp-contract=off",
           "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", "-o", OUT, SRC]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
