"""Guided-mode / plasmon pole-residue extraction on the deformed contour, through the C ABI,
against the oracle's dense real-axis integral (Cauchy: with lossy layers every pole lies above
the real axis, so the contour integral equals the real-axis one over the same end points).

Geometry of the 3-layer dipole problem: vertical dipole 20 nm above a 50 nm uniaxial film
(εe = 4+0.2i) on glass, λ = 600 nm, contour kρ = t - 0.05 i k0 sin(π t / 20 k0) with panel
breaks at the half-space light lines, G on 24 radii (6-3000 nm) x 9 heights (0-200 nm)."""
import numpy as np
import pytest

from helpers import relerr
from yellowthinfilms_b200.materials import FlatOpticalLayer, IsotropicMaterial, UniaxialMaterial

pytestmark = pytest.mark.gpu

K0 = 2 * np.pi / 600.0
RHO = np.geomspace(6.0, 3000.0, 24)
ZO = np.linspace(0.0, 200.0, 9)


def _stack(eo):
    return [FlatOpticalLayer(IsotropicMaterial(1.0), 200.0), FlatOpticalLayer(UniaxialMaterial(eo, 4.0 + 0.2j), 50.0),
            FlatOpticalLayer(IsotropicMaterial(2.25), 100.0)]


def _real_axis_oracle(oracle, st):
    lines = sorted({float(x) for L in st for x in oracle.light_lines(L, K0, 0.0) if 0 < x < 20 * K0})
    sing = sorted({float(x) for L in (st[0], st[-1]) for x in oracle.light_lines(L, K0, 0.0)})
    brk = [0.0] + lines + [20 * K0]
    panels = []
    for a, b in zip(brk[:-1], brk[1:]):
        n = max(8, int(np.ceil(6000 * (b - a) / (20 * K0))))
        e = np.linspace(a, b, n + 1)
        panels += list(zip(e[:-1], e[1:]))
    kr, wr = oracle.gl_rule(panels, 8, singular=sing)
    oc = oracle.build_cavity_transfer_1d(st, K0, 1, kr, wr, obs_layers=[1])
    return oracle.closed_form_G(oc, 1, 20.0, ZO, RHO, [0.0])


def _setup(st):
    from yellowthinfilms_b200 import api, poles as PL
    sto = api.Stack(st)
    bps = sorted({float(x) for L in (st[0], st[-1]) for x in api.layer_light_lines(L, K0)})
    _, _, info = api.point_kx_grid(sto, K0, 1, h_min=20.0, rho_max=3000.0, kr_cap=20 * K0, rtol=1e-11)
    probe = dict(obs_layer=1, zsrc=20.0, z_obs=[0.0, 100.0], xs=[6.0, 300.0], ys=[0.0])
    poles = PL.contour_poles(sto, K0, 1, info["poles"], probe, branch_points=bps)
    return sto, bps, poles


def _contour_G(st, bps, npan, poles):
    from yellowthinfilms_b200 import api, poles as PL
    k, w = api.contour_rule(K0, npanels=npan, order=8, breaks=bps)
    c = api.build_cavity_transfer_1d_contour(st, K0, 1, k, w, obs_layers=[1])
    return PL.closed_form_G_contour(c, 1, 20.0, ZO, RHO, [0.0], poles=poles), len(k)


def test_extracting_a_sharp_guided_mode_needs_fewer_nodes(oracle):
    """In-plane film loss 0.01: a guided mode at k_p ≈ (2.408 + 0.015i) k0 sits 0.02 k0 above
    the path. The contour alone is still above 1e-6 with 128 panels; with the poles extracted
    64 panels (half the nodes) are within 1e-6 of the oracle, and the residue of each pole does
    not depend on the circle it is taken on (the integrand is analytic around it)."""
    from yellowthinfilms_b200 import poles as PL
    st = _stack(-3.0 + 0.01j)
    Go = _real_axis_oracle(oracle, st)
    sto, bps, poles = _setup(st)
    assert any(abs(kp.real / K0 - 2.408) < 0.01 and 0 < kp.imag / K0 < 0.03 for kp, _ in poles), poles
    G128, n128 = _contour_G(sto, bps, 128, ())
    G64p, n64 = _contour_G(sto, bps, 64, poles)
    assert relerr(G128, Go) > 1e-6
    assert relerr(G64p, Go) < 1e-6 and n64 < n128
    assert relerr(G64p[..., 2, 2], Go[..., 2, 2]) < 1e-6
    R1 = PL.residues(sto, K0, 1, poles, 1, 20.0, ZO[:3], RHO[:5], [0.0])
    R2 = PL.residues(sto, K0, 1, [(kp, 0.5 * r) for kp, r in poles], 1, 20.0, ZO[:3], RHO[:5], [0.0])
    for a, b in zip(R1, R2):
        assert relerr(a, b) < 1e-8


def test_extraction_on_the_problem_film_is_harmless(oracle):
    """The problem's own film (εo = -3+0.4i): its guided mode is broad (Γ ≈ 0.19 k0), the
    contour alone reaches 1e-6 with 64 panels and extracting the pole changes G by far less."""
    st = _stack(-3.0 + 0.4j)
    Go = _real_axis_oracle(oracle, st)
    sto, bps, poles = _setup(st)
    G0, _ = _contour_G(sto, bps, 64, ())
    Gp, _ = _contour_G(sto, bps, 64, poles)
    assert relerr(G0, Go) < 1e-6 and relerr(Gp, Go) < 1e-6
    assert relerr(Gp, G0) < 1e-7
