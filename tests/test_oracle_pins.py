"""Pins of the CPU oracle against the reference's golden data and known answers.

Each test restates a check of the reference's own validation scripts (cited per test);
none needs a GPU. The oracle is the checker of the CUDA path, so it is pinned first.
"""
import json
import os

import numpy as np
import pytest

from helpers import (FOUNDATION_STACKS, e_free, krho_grid, lay, m_bi, m_biT, m_gl, m_gyr, m_uni, m_vac, relerr,
                     uniform_phi)
from yellowthinfilms_b200.materials import (BiaxialMaterial, FlatLayer, FlatOpticalLayer, GyrotropicMaterial,
                                            IsotropicMaterial, UniaxialMaterial)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("case", ["film", "stack"])
def test_reflectance_matches_committed_golden(oracle, case):
    """comparisons/gila_airy/results/{film,stack}.tsv: R_own of own_reflectance
    (airy_comparison.jl:66-82), to the 10 printed decimals."""
    g = json.load(open(os.path.join(GOLDEN, f"reflectance_{case}.json")))
    vac = FlatOpticalLayer(IsotropicMaterial(1.0), 0.0)
    st = [vac] + [FlatOpticalLayer(IsotropicMaterial(1 + complex(a, b)), d) for a, b, d in g["films_chi_re_im_d"]] + [vac]
    worst = max(abs(oracle.own_reflectance(st, 2 * np.pi, r["angle"], r["pol"]) - r["R_own"]) for r in g["rows"])
    assert worst < 6e-11


def _tmm(films, th, pol, k0=2 * np.pi):
    """Characteristic-matrix reflectance (airy_comparison.jl:35-50), written independently."""
    kx = k0 * np.sin(np.radians(th))
    kz0 = k0 * np.cos(np.radians(th))
    eta = (lambda e, kz: kz / k0) if pol == "s" else (lambda e, kz: e * k0 / kz)
    e0 = eta(1.0, kz0)
    M = np.eye(2, dtype=complex)
    for chi, d in films:
        e = 1 + chi
        kz = np.sqrt(complex(e * k0 ** 2 - kx ** 2))
        dl, ej = kz * d, eta(e, kz)
        M = M @ np.array([[np.cos(dl), -1j * np.sin(dl) / ej], [-1j * ej * np.sin(dl), np.cos(dl)]])
    num = e0 * M[0, 0] + e0 ** 2 * M[0, 1] - M[1, 0] - e0 * M[1, 1]
    den = e0 * M[0, 0] + e0 ** 2 * M[0, 1] + M[1, 0] + e0 * M[1, 1]
    return abs(num / den) ** 2


def test_reflectance_vs_transfer_matrix(oracle):
    films = [(1.25, 0.25), (3.0, 3 / 16), (1.0 + 0.1j, 1 / 8)]
    vac = FlatOpticalLayer(IsotropicMaterial(1.0), 0.0)
    st = [vac] + [FlatOpticalLayer(IsotropicMaterial(1 + c), d) for c, d in films] + [vac]
    for pol in "sp":
        for th in (0.0, 17.5, 45.0, 72.5, 85.0):
            assert abs(oracle.own_reflectance(st, 2 * np.pi, th, pol) - _tmm(films, th, pol)) < 1e-13


def test_foundation_transfer_map_vs_modal_amp(oracle):
    """Gz_ClosedForm_Foundation_Validation.jl: T^o·[S₊;S₋] vs Modal_amp (cross-layer) and
    Modal_amp_profile's reflected part (same layer), < 1e-11."""
    w = 2 * np.pi
    kts = [(0.3, 0.0), (1.2, 0.4), (2.9, -1.1), (8.0, 3.0)]
    worst_c = worst_s = 0.0
    for _, st in FOUNDATION_STACKS:
        N = len(st)
        for kx, ky in kts:
            for layer in range(1, N):
                d = st[layer - 1].d
                for q in range(3):
                    for zf in (0.13, 0.5, 0.91):
                        tu, ref, sn = oracle.foundation(st, w, kx, ky, layer, q, zf * d)
                        for o in range(1, N + 1):
                            if o == layer:
                                worst_s = max(worst_s, np.linalg.norm(tu[o - 1] - ref[o - 1]) / max(sn, 1e-300))
                            else:
                                worst_c = max(worst_c, relerr(tu[o - 1], ref[o - 1]))
    assert worst_c < 1e-11 and worst_s < 1e-11


@pytest.mark.parametrize("idx", range(len(FOUNDATION_STACKS)))
def test_modes_are_eigenpairs_of_berreman(oracle, idx):
    """Every sorted mode (V, Q) satisfies B·V = Q·V for its layer's Berreman matrix
    (mod_ModeSolver.jl:122-193, 243-265); W = R4s·V (mod_ModeSolver.jl:278)."""
    _, st = FOUNDATION_STACKS[idx]
    w = 2 * np.pi
    for kx, ky in [(0.3, 0.0), (1.2, 0.4), (8.0, 3.0)]:
        modes = oracle.modes_stack(st, w, kx, ky)
        for l, m in zip(st, modes):
            B = oracle.berreman(l, w, kx, ky)
            for V, Q, W in ((m["Vf"], m["Qf"], m["Wf"]), (m["Vb"], m["Qb"], m["Wb"])):
                for j in range(2):
                    r = B @ V[:, j] - Q[j] * V[:, j]
                    assert np.linalg.norm(r) < 1e-10 * max(1, abs(Q[j])) * np.linalg.norm(V[:, j])
                    assert np.allclose(W[:, j], [V[3, j], -V[2, j], -V[1, j], V[0, j]])


def test_general_modes_match_numpy_eigen(oracle):
    """The general path's eigenvalues are LAPACK's (compare numpy's geev)."""
    st = FOUNDATION_STACKS[4][1]
    w = 2 * np.pi
    modes = oracle.modes_stack(st, w, 1.2, 0.4)
    B = oracle.berreman(st[0], w, 1.2, 0.4)
    ev = np.sort_complex(np.linalg.eigvals(B))
    got = np.sort_complex(np.concatenate([modes[0]["Qf"], modes[0]["Qb"]]))
    assert np.allclose(ev, got, rtol=1e-12, atol=1e-12)


def test_gauss_legendre_correctly_rounded(oracle):
    """The oracle's Gauss–Legendre rule (FastGaussQuadrature.gausslegendre's role,
    mod_KxGrid.jl:362) is within 1 ulp of the exact nodes and weights (mpmath, 40 digits);
    scipy agrees to 1e-14."""
    import mpmath as mp
    from scipy.special import roots_legendre
    mp.mp.dps = 40
    for n in (4, 8, 12, 16):
        x, w = oracle.gauss_legendre(n)
        xs, ws = roots_legendre(n)
        assert np.allclose(x, xs, rtol=0, atol=1e-14) and np.allclose(w, ws, rtol=1e-13, atol=0)
        assert np.all(np.diff(x) > 0)
        for i in range(n):
            r = mp.findroot(lambda t: mp.legendre(n, t), x[i])
            dp = mp.diff(lambda t: mp.legendre(n, t), r)
            we = 2 / ((1 - r ** 2) * dp ** 2)
            assert abs(mp.mpf(x[i]) - r) <= np.spacing(max(abs(x[i]), 1e-300)) or (x[i] == 0 and abs(r) < 1e-30)
            assert abs(mp.mpf(w[i]) - we) <= np.spacing(w[i])


def test_light_lines_closed_forms(oracle):
    """Gz_ClosedForm_Quadrature_Validation.jl:49-64 ([L]), 1e-12 relative to ω."""
    w = 2 * np.pi
    ll = lambda m, mu=None: oracle.light_lines(FlatOpticalLayer(m, 1.0) if mu is None else FlatLayer(m, mu, 1.0), w, 0.0)
    e = abs(ll(IsotropicMaterial(2.25 + 0.01j))[0] - w * np.sqrt(2.25 + 0.01j).real)
    et, ez, mt, mz = 3 + 0.1j, -2 + 0.1j, 1.6 + 0.05j, 0.7 + 0.05j
    L = ll(UniaxialMaterial(et, ez), UniaxialMaterial(mt, mz))
    assert len(L) == 1
    e = max(e, abs(L[0] - w * np.sqrt(et * mz).real))
    L = ll(IsotropicMaterial(2.25), IsotropicMaterial(1.5))
    e = max(e, abs(L[0] - w * np.sqrt(2.25 * 1.5)))
    e1, g, e3 = 1.0, 0.3, 2.0
    vg = GyrotropicMaterial([[e1, 0, 1j * g], [0, e3, 0], [-1j * g, 0, e1]])
    Lx = oracle.light_lines(FlatOpticalLayer(vg, 1.0), w, 0.0)
    Ly = oracle.light_lines(FlatOpticalLayer(vg, 1.0), w, np.pi / 2)
    e = max(e, np.max(np.abs(Lx - np.sort(w * np.sqrt([(e1 ** 2 - g ** 2) / e1, e3])))),
            np.max(np.abs(Ly - np.sort(w * np.sqrt([e1 - g, e1 + g])))))
    assert e / w < 1e-12


def test_material_class(oracle):
    """Gz_ClosedForm_Quadrature_Validation.jl:65-70."""
    def lorentz(nu, einf, TO, LO, gam):
        return einf * (1 + (LO ** 2 - TO ** 2) / (TO ** 2 - nu ** 2 - 1j * nu * gam))
    hbn = lambda nu: UniaxialMaterial(lorentz(nu, 4.99, 1361.0, 1614.0, 1.0), lorentz(nu, 2.94, 760.5, 825.0, 1.0))
    vg = GyrotropicMaterial([[1, 0, 0.3j], [0, 2, 0], [-0.3j, 0, 1]])
    mats = [IsotropicMaterial(2.25 + 0.01j), IsotropicMaterial(-20.0 + 1j), hbn(1500.0), hbn(812.0), vg,
            GyrotropicMaterial([[2, 0.5, 0], [0.5, -3, 0], [0, 0, 1]])]
    want = ["dielectric", "metallic", "hyperbolic", "hyperbolic", "gyrotropic", "hyperbolic"]
    assert [oracle.material_class(FlatOpticalLayer(m, 1.0)) for m in mats] == want


@pytest.mark.parametrize("omega", [2 * np.pi, np.pi, 1.0, 3.7])
def test_free_space_dipole_normalization(oracle, omega):
    """Gz_ClosedForm_Point_Validation.jl [f]: near-vacuum stack vs the analytic dipole,
    1D and 2D caches (catches an ω/2π factor). The fixed rule here is converged to
    ~4e-8; the reference's adaptive engine reaches 1e-10."""
    ef = 1.0 + 1e-4j
    st = [lay(IsotropicMaterial(ef), 3.0) for _ in range(3)]
    zs, zo, x = 1.0, 1.7, 0.4
    kx, wt, _ = oracle.fixed_grid_1d(st, omega, 2, h_min=0.025, rho_max=1.0, scan=False, rtol=1e-10)
    Gref = np.stack([e_free(np.array([x, 0, zo - zs]), np.eye(3)[q].astype(complex), omega * np.sqrt(ef), ef)
                     for q in range(3)], axis=1)
    c1 = oracle.build_cavity_transfer_1d(st, omega, 2, kx, wt)
    G1 = oracle.closed_form_G(c1, 2, zs, [zo], [x], [0.0])[0, 0, 0]
    ph, wp = uniform_phi(48)
    c2 = oracle.build_cavity_transfer_2d(st, omega, 2, kx, wt, ph, wp, obs_layers=[2])
    G2 = oracle.closed_form_G(c2, 2, zs, [zo], [x], [0.0])[0, 0, 0]
    assert relerr(G1, Gref) < 1e-7 and relerr(G2, Gref) < 1e-7


def test_rotation_fill_equals_full_solve_and_1d(oracle):
    """Gz_ClosedForm_Point_Validation.jl [c]: 2D rotation fill = full per-node solve = 1D
    path on the same kρ nodes, < 1e-10 (one source layer, three obs layers)."""
    w = 2 * np.pi
    st = [lay(m_vac, 1.0), lay(m_uni, 0.8), lay(m_gl, 0.5), lay(m_vac, 1.0)]
    kr, wr = krho_grid(st, w, kmax=12.0, width=1.0)
    ph, wp = uniform_phi(16)
    x5 = np.arange(-0.2, 0.21, 0.1)
    worst = 0.0
    for src in (1, 2):
        cr = oracle.build_cavity_transfer_2d(st, w, src, kr, wr, ph, wp)
        cf = oracle.build_cavity_transfer_2d(st, w, src, kr, wr, ph, wp, rotation=False)
        c1 = oracle.build_cavity_transfer_1d(st, w, src, kr, wr)
        zs = 0.4 * st[src - 1].d
        for obs in (1, 2, 3):
            zo = [0.05 * st[obs - 1].d, 0.95 * st[obs - 1].d] if obs == src else [0.3 * st[obs - 1].d]
            Gr = oracle.closed_form_G(cr, obs, zs, zo, x5, x5)
            worst = max(worst, relerr(Gr, oracle.closed_form_G(cf, obs, zs, zo, x5, x5)),
                        relerr(oracle.closed_form_G(c1, obs, zs, zo, x5, x5), Gr))
    # the 1D path's Jacobi-Anger sum equals the 2D trapezoid in φ only when N_φ resolves
    # e^{i kρ ρ cos φ}: at kρ·ρ ≤ 12·0.29 and N_φ = 16 the trapezoid error is ~1e-11
    assert worst < 1e-9


def test_reciprocity(oracle):
    """Gz_ClosedForm_Point_Validation.jl [e]: G₂₃(r←r') = G₃₂(r'←r)ᵀ, isotropic (1D) and
    biaxial (2D), < 1e-10."""
    w = 2 * np.pi
    ph, wp = uniform_phi(48)
    worst = 0.0
    for mat, use2d in ((m_gl, False), (m_bi, True)):
        st = [lay(m_vac, 1.0), lay(mat, 0.7), lay(m_gl, 0.6), lay(m_vac, 1.0)]
        kr, wr = krho_grid(st, w, kmax=15.0)
        if use2d:
            c2 = oracle.build_cavity_transfer_2d(st, w, 2, kr, wr, ph, wp)
            c3 = oracle.build_cavity_transfer_2d(st, w, 3, kr, wr, ph, wp)
        else:
            c2 = oracle.build_cavity_transfer_1d(st, w, 2, kr, wr)
            c3 = oracle.build_cavity_transfer_1d(st, w, 3, kr, wr)
        z2, z3 = 0.45, 0.2
        for dx, dy in ((0.0, 0.0), (0.3, 0.0), (0.2, -0.25)):
            G23 = oracle.closed_form_G(c2, 3, z2, [z3], [dx], [dy])[0, 0, 0]
            G32 = oracle.closed_form_G(c3, 2, z3, [z2], [-dx], [-dy])[0, 0, 0]
            worst = max(worst, np.linalg.norm(G23 - G32.T) / np.linalg.norm(G23))
    assert worst < 1e-10


def test_rotation_covariance(oracle):
    """Gz_ClosedForm_Point_Validation.jl [d]: G_B(R r) = R G_A(r) Rᵀ, biaxial
    diag(a,b,c) → diag(b,a,c) and a gyrotropic medium invariant under R, < 1e-10."""
    w = 2 * np.pi
    xo = np.arange(-0.4, 0.41, 0.2)
    No = len(xo)
    R = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    ph, wp = uniform_phi(48)
    worst = 0.0
    for A, B in ((m_bi, m_biT), (m_gyr, m_gyr)):
        stA = [lay(m_vac, 1.0), lay(A, 0.7), lay(m_gl, 0.5), lay(m_vac, 1.0)]
        stB = [lay(m_vac, 1.0), lay(B, 0.7), lay(m_gl, 0.5), lay(m_vac, 1.0)]
        kr, wr = krho_grid(stA, w, kmax=15.0)
        cA = oracle.build_cavity_transfer_2d(stA, w, 2, kr, wr, ph, wp)
        cB = oracle.build_cavity_transfer_2d(stB, w, 2, kr, wr, ph, wp)
        for obs, zo in ((2, 0.1), (1, 0.8), (3, 0.25)):
            GA = oracle.closed_form_G(cA, obs, 0.35, [zo], xo, xo)
            GB = oracle.closed_form_G(cB, obs, 0.35, [zo], xo, xo)
            err = max(np.linalg.norm(GB[No - 1 - j, i, 0] - R @ GA[i, j, 0] @ R.T) for i in range(No) for j in range(No))
            worst = max(worst, err / max(np.linalg.norm(GA[i, j, 0]) for i in range(No) for j in range(No)))
    assert worst < 1e-10


def test_mlp_reference_gradient_matches_finite_differences():
    """The FP64 MLP restatement (the checker of the GPU training kernels) differentiates its
    own loss correctly: central differences at unrounded weights."""
    import ytf_mlp_ref as R
    rng = np.random.default_rng(3)
    sizes = [7, 9, 8, 2]
    n = sum(sizes[i] * sizes[i + 1] + sizes[i + 1] for i in range(len(sizes) - 1))
    p = rng.normal(0, 0.5, n)
    X = rng.normal(0, 1, (5, 7))
    T = np.stack([rng.normal(0, 1, 5), rng.uniform(0, 1, 5)], 1)
    _, g = R.loss_and_grad(p, sizes, X, T, round_weights=False)
    h = 1e-6
    fd = np.zeros(n)
    for i in range(n):
        e = np.zeros(n); e[i] = h
        fd[i] = (R.loss_and_grad(p + e, sizes, X, T, False)[0] - R.loss_and_grad(p - e, sizes, X, T, False)[0]) / (2 * h)
    assert np.max(np.abs(fd - g)) < 1e-7 * max(1.0, np.max(np.abs(g)))
