"""The C-ABI library: loads without a GPU, exports every symbol include/ytf.h declares,
and its host-side pieces agree with the oracle (no GPU calls here)."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "ytf.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ytf_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    from yellowthinfilms_b200 import build, _native
    path = build.build()
    L = ctypes.CDLL(path)
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_native.SIGNATURES), set(names) ^ set(_native.SIGNATURES)
    assert L.ytf_version() >= 10000


def test_host_gauss_legendre_bitexact_with_oracle(oracle):
    from yellowthinfilms_b200 import api
    for n in (1, 2, 3, 5, 8, 12, 16, 24):
        x, w = api.gausslegendre(n)
        xo, wo = oracle.gauss_legendre(n)
        assert np.array_equal(x, xo) and np.array_equal(w, wo), n


def test_no_gpu_context_fails_loudly():
    """Without a CUDA device the product raises instead of falling back to the CPU."""
    import torch
    if torch.cuda.is_available():
        return
    from yellowthinfilms_b200 import api
    import pytest
    with pytest.raises(RuntimeError):
        api.Context(0)


def test_host_light_lines_bit_exact_with_oracle(oracle):
    """libytf's host light lines (ytf_layer_light_lines: the k-grid's panel breaks) equal the
    oracle's bit for bit, for every layer of the test stacks and the bench stack, several
    frequencies and azimuths (no GPU needed)."""
    import bench
    from helpers import FOUNDATION_STACKS
    from yellowthinfilms_b200 import api
    stacks = [s for _, s in FOUNDATION_STACKS] + [bench.make_stack()]
    n = 0
    for st in stacks:
        for L in st:
            for w in (1.0, 2 * np.pi, 0.0104719755, 3.7):
                for phi in (0.0, 0.3, 1.2):
                    a = api.layer_light_lines(L, w, phi)
                    b = np.asarray(oracle.light_lines(L, w, phi))
                    assert len(a) == len(b) and np.array_equal(a, b), (a, b)
                    n += 1
    assert n > 300


def test_halve_panels_array_form_equals_pair_form():
    """halve_panels on a [n, 2] array gives the pair form's panels bit for bit (the batched
    refinement levels pass arrays); mod_KxGrid.jl:387-388."""
    from yellowthinfilms_b200 import api
    rng = np.random.default_rng(3)
    e = np.sort(rng.uniform(0.0, 7.0, 41))
    pairs = list(zip(e[:-1], e[1:]))
    arr = api.halve_panels(np.array(pairs))
    lst = api.halve_panels(pairs)
    assert arr.shape == (80, 2)
    assert np.array_equal(arr, np.array(lst))
    assert np.array_equal(api.halve_panels(arr), np.array(api.halve_panels(lst)))


def test_noalloc_wrapper_refuses_host_tensors_and_wrong_dtypes():
    """closed_form_G_noalloc hands raw addresses to the library, so it must refuse a host
    tensor (the kernels would read a host address) and a complex64 output (the reduction
    would write twice its size) before any call."""
    import pytest
    import torch
    from yellowthinfilms_b200 import api
    z = torch.zeros(2, dtype=torch.float64)
    out = torch.zeros(2 * 2 * 2 * 9, dtype=torch.complex128)
    with pytest.raises(api.YTFError, match="must be on cuda:0"):
        api._noalloc_tensors(0, z, z, z, out)
    meta = lambda dt: torch.empty(2 * 2 * 2 * 9, dtype=dt, device="meta")
    with pytest.raises(api.YTFError, match="must be"):
        api._noalloc_tensors(0, z, z, z, meta(torch.complex64))
    with pytest.raises(api.YTFError, match="must be a torch tensor"):
        api._noalloc_tensors(0, np.zeros(2), z, z, out)
