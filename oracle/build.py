"""Build recipe of the CPU oracle (test infrastructure only).

Compiles ``oracle/ytf_oracle.cpp`` into ``oracle/_build/libytf_oracle.so`` with plain g++
and OpenMP. No contraction of a*b+c into FMA (``-ffp-contract=off``), so the oracle's node
construction is reproducible bit for bit; complex arithmetic follows Fortran rules (the
textbook formulas, as Julia's ``*`` and ``/`` for ComplexF64 on finite values).

Usage: ``python oracle/build.py`` (idempotent; rebuilds when the source is newer).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "ytf_oracle.cpp")
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "libytf_oracle.so")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
           "-fcx-fortran-rules", "-o", OUT + ".tmp", SRC]
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
