"""Build libytf.so in-tree for sm_100a (B200).

    python -m yellowthinfilms_b200.build [--force]

Every ``csrc/*.cu`` is compiled to its own object file (in parallel, one nvcc per source;
a source is recompiled only when it or a header is newer than its object) and the objects
are linked into ``yellowthinfilms_b200/_build/libytf.so`` (git-ignored, but it travels with
the source tree). No device code crosses a source file, so no relocatable device code is
needed. The CUDA runtime is linked statically, so the library needs only the driver.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libytf.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
    # host complex arithmetic without the C99 Annex-G NaN recovery and without contraction,
    # as the oracle build: the host-side k-grid (light lines, panels) then agrees bit for bit
    "-Xcompiler", "-fcx-fortran-rules", "-Xcompiler", "-ffp-contract=off",
    "-diag-suppress", "177",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _obj(src):
    return os.path.join(OUT_DIR, os.path.splitext(os.path.basename(src))[0] + ".o")


def _newer(deps, target) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    hdr = _headers()
    todo = [s for s in sources() if force or _newer([s] + hdr, _obj(s))]

    def compile_one(src):
        cmd = [nvcc, *NVCC_FLAGS, "-I", INCLUDE, "-c", "-o", _obj(src) + ".tmp", src]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        os.replace(_obj(src) + ".tmp", _obj(src))

    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        list(ex.map(compile_one, todo))
    objs = [_obj(s) for s in sources()]
    if force or todo or _newer(objs, LIB):
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp", *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
