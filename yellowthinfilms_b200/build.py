"""Build libytf.so in-tree for sm_100a (B200).

    python -m yellowthinfilms_b200.build [--force]

One nvcc invocation over every ``csrc/*.cu``; the result lands in
``yellowthinfilms_b200/_build/libytf.so`` (git-ignored, but it travels with the source
tree). The CUDA runtime is linked statically, so the library needs only the driver.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libytf.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    # host complex arithmetic without the C99 Annex-G NaN recovery and without contraction,
    # as the oracle build: the host-side k-grid (light lines, panels) then agrees bit for bit
    "-Xcompiler", "-fcx-fortran-rules", "-Xcompiler", "-ffp-contract=off",
    "-diag-suppress", "177",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, "-I", INCLUDE, "-o", LIB + ".tmp", *sources()]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
