"""The allocation-free synthesis entry point, ytf_green_noalloc, through the C ABI.

Hosts that keep every device byte in their own pool (a Julia CUDA.jl session, a caching
allocator), or that cannot afford cudaMalloc's device-wide synchronisation, call this
variant: its scratch is a fixed array inside the library instead of memory the library
allocates. Its result must equal the allocating entry point's (closed_form_G, same
cache) to the FP64 parity tolerance of the other GPU tests, on two calls in a row (the
second call finds the first call's leftovers in the shared array), and a request beyond
the fixed size must be refused with a clear error. This file is collected last.
"""
import numpy as np
import pytest

from helpers import FOUNDATION_STACKS, krho_grid, relerr, uniform_phi

pytestmark = pytest.mark.gpu

W = 2 * np.pi


def test_noalloc_green_matches_allocating_entry_point_on_two_calls():
    import torch
    from yellowthinfilms_b200 import api
    _, st = FOUNDATION_STACKS[3]  # biaxial: the general eigen path
    kr, wr = krho_grid(st, W, kmax=10.0, width=1.0)
    ph, wp = uniform_phi(8)
    cache = api.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp, obs_layers=[1, 2, 3])
    dev = torch.device("cuda", cache.ctx.device)
    calls = [(2, 0.3, [0.1, 0.4, 0.7], np.linspace(-0.3, 0.3, 5), np.linspace(-0.2, 0.25, 4), "all"),
             (3, 0.3, [0.05, 0.2], np.linspace(-0.1, 0.4, 3), np.array([0.0, 0.15]), "all")]
    for obs, zs, zo, xs, ys, terms in calls:
        ref = api.closed_form_G(cache, obs, zs, zo, xs, ys, terms=terms)
        t = lambda a: torch.tensor(np.asarray(a, dtype=np.float64), device=dev)
        out = torch.empty(len(xs) * len(ys) * len(zo) * 9, dtype=torch.complex128, device=dev)
        api.closed_form_G_noalloc(cache, obs, zs, t(zo), t(xs), t(ys), out, terms=terms)
        got = out.cpu().numpy().reshape(3, 3, len(zo), len(ys), len(xs)).transpose(4, 3, 2, 1, 0)
        assert relerr(got, ref) < 1e-10, relerr(got, ref)


def test_noalloc_refuses_requests_beyond_its_fixed_scratch():
    import torch
    from yellowthinfilms_b200 import api
    _, st = FOUNDATION_STACKS[3]
    kr, wr = krho_grid(st, W, kmax=10.0, width=1.0)
    ph, wp = uniform_phi(8)
    cache = api.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp, obs_layers=[2])
    dev = torch.device("cuda", cache.ctx.device)
    nx = ny = 800  # 9 * nz * (nodes + 640000) > 4,194,304
    xs = torch.zeros(nx, dtype=torch.float64, device=dev)
    zo = torch.tensor([0.2], dtype=torch.float64, device=dev)
    out = torch.empty(nx * ny * 9, dtype=torch.complex128, device=dev)
    with pytest.raises(api.YTFError, match="exceed the fixed scratch"):
        api.closed_form_G_noalloc(cache, 2, 0.3, zo, xs, xs, out)
