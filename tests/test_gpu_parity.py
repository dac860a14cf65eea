"""GPU parity: the CUDA path (through the C ABI) against the FP64 oracle on identical
nodes. FP64 synthesis: ≤ 1e-10 relative (norm over the array, the reference's relerr);
the per-node cache to 1e-9; k-grid construction bit-exact."""
import numpy as np
import pytest

from helpers import (FOUNDATION_STACKS, e_free, krho_grid, lay, m_bi, m_biT, m_gl, m_gyr, m_gyr4, m_uni, m_vac, relerr,
                     uniform_phi)
from yellowthinfilms_b200.materials import IsotropicMaterial, UniaxialMaterial

pytestmark = pytest.mark.gpu

W = 2 * np.pi


@pytest.fixture(scope="module")
def ytf():
    from yellowthinfilms_b200 import api
    return api


def config1_stack(d_air=200.0):
    """Air / uniaxial film (εo = -3+0.4i, εe = 4+0.2i, 50 nm) / glass 2.25 (nm units)."""
    return [lay(IsotropicMaterial(1.0), d_air), lay(UniaxialMaterial(-3.0 + 0.4j, 4.0 + 0.2j), 50.0),
            lay(IsotropicMaterial(2.25), 100.0)]


def _cmp_cache(gc, oc, tol=1e-9):
    g, o = gc.export(), oc.export()
    vg, tg, _ = gc.status()
    assert np.array_equal(vg, o["valid"])
    assert np.array_equal(tg, o["Tvalid"])
    for key in ("Qf", "Qb"):
        assert relerr(g[key], o[key]) < tol, key
    # seeds and T depend on the per-mode normalisation only through a phase; compare
    # the observable combination T·[sf; sb] per node
    for i in range(len(gc.obs_layers)):
        ug = np.einsum("nij,njq->niq", g["T"][i][:, :, :2], g["sf"]) + np.einsum("nij,njq->niq", g["T"][i][:, :, 2:], g["sb"])
        uo = np.einsum("nij,njq->niq", o["T"][i][:, :, :2], o["sf"]) + np.einsum("nij,njq->niq", o["T"][i][:, :, 2:], o["sb"])
        eg = np.einsum("nfm,nmq->nfq", g["basis"][i][:, 0:3], ug[:, :2]) + np.einsum("nfm,nmq->nfq", g["basis"][i][:, 3:6], ug[:, 2:])
        eo = np.einsum("nfm,nmq->nfq", o["basis"][i][:, 0:3], uo[:, :2]) + np.einsum("nfm,nmq->nfq", o["basis"][i][:, 3:6], uo[:, 2:])
        assert relerr(eg, eo) < tol


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_transfer_1d_cache_matches_oracle(ytf, oracle, idx):
    _, st = FOUNDATION_STACKS[idx]
    kx, wt = krho_grid(st, W, kmax=15.0)
    for src in range(1, len(st)):
        gc = ytf.build_cavity_transfer_1d(st, W, src, kx, wt)
        oc = oracle.build_cavity_transfer_1d(st, W, src, kx, wt)
        _cmp_cache(gc, oc)


@pytest.mark.parametrize("idx", [1, 3, 4])
def test_source_only_chain_matches_general_chain(ytf, oracle, idx):
    """A cache whose only observation layer is the source layer takes the forward-only
    chain (SRight[src] accumulated left to right, no stored interfaces); the same node
    solve with every layer observed takes the general chain (backward SRight scan). The
    source-layer rows must agree (to rounding: the star products are grouped differently),
    and the fast-path cache must match the oracle, for top, middle and last finite source
    layers, 1D and 2D."""
    _, st = FOUNDATION_STACKS[idx]
    kr, wr = krho_grid(st, W, kmax=12.0)
    ph, wp = uniform_phi(4)
    N = len(st)
    two_d = idx >= 3
    for src in sorted({1, max(1, N // 2), N - 1}):
        if two_d:
            fast = ytf.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp, obs_layers=[src])
            full = ytf.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp, obs_layers=list(range(1, N + 1)))
            oc = oracle.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp, obs_layers=[src])
        else:
            fast = ytf.build_cavity_transfer_1d(st, W, src, kr, wr, obs_layers=[src])
            full = ytf.build_cavity_transfer_1d(st, W, src, kr, wr, obs_layers=list(range(1, N + 1)))
            oc = oracle.build_cavity_transfer_1d(st, W, src, kr, wr, obs_layers=[src])
        gf, gg = fast.export(), full.export()
        i = full.obs_layers.index(src)
        assert relerr(gf["T"][0], gg["T"][i]) < 1e-11, src
        for key in ("Qf", "Qb", "sf", "sb"):
            assert relerr(gf[key], gg[key]) < 1e-13, (src, key)
        assert relerr(gf["basis"][0], gg["basis"][i]) < 1e-13, src
        assert np.array_equal(fast.status()[0], full.status()[0])
        _cmp_cache(fast, oc)


def deep_stack(n_layers=24):
    """Vacuum / alternating gyrotropic, transposed-biaxial, uniaxial and glass films / vacuum:
    more than 16 layers, so the mode-matching swaps of layers 16 and up sit past bit 31 of
    the per-node swap mask."""
    films = [m_gyr4, m_biT, m_uni, m_gl]
    st = [lay(m_vac, 0.5)]
    for i in range(n_layers - 2):
        st.append(lay(films[i % 4], 0.12 + 0.01 * (i % 3)))
    st.append(lay(m_vac, 0.5))
    return st


@pytest.mark.gpu
def test_source_only_chain_deep_stack(ytf, oracle):
    """24-layer stack, source layers on both sides of layer 16: the forward-only chain agrees
    with the general chain and with the oracle."""
    st = deep_stack(24)
    kr, wr = krho_grid(st, W, kmax=5.0, width=1.0, order=6)
    ph, wp = uniform_phi(3)
    N = len(st)
    for src in (3, 18, N - 1):
        fast = ytf.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp, obs_layers=[src])
        full = ytf.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp, obs_layers=list(range(1, N + 1)))
        oc = oracle.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp, obs_layers=[src])
        gf, gg = fast.export(), full.export()
        i = full.obs_layers.index(src)
        assert relerr(gf["T"][0], gg["T"][i]) < 1e-10, src
        for key in ("Qf", "Qb", "sf", "sb"):
            assert relerr(gf[key], gg[key]) < 1e-12, (src, key)
        assert np.array_equal(fast.status()[0], full.status()[0])
        _cmp_cache(fast, oc)


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_green_1d_matches_oracle(ytf, oracle, idx):
    _, st = FOUNDATION_STACKS[idx]
    kx, wt = krho_grid(st, W, kmax=15.0)
    xs = np.array([-0.3, 0.0, 0.2, 0.45])
    ys = np.array([0.0, 0.15, -0.25])
    N = len(st)
    for src in range(1, N):
        gc = ytf.build_cavity_transfer_1d(st, W, src, kx, wt)
        oc = oracle.build_cavity_transfer_1d(st, W, src, kx, wt)
        zs = 0.4 * st[src - 1].d
        for obs in range(1, N + 1):
            d = st[obs - 1].d
            zo = [0.1 * d, 0.4 * d, 0.75 * d] if obs != src else [0.05 * d, 0.4 * d, 0.95 * d]
            terms_list = ["all", "scattered", "direct", "toeplitz", "hankel"] if obs == src else ["all"]
            for terms in terms_list:
                G = ytf.closed_form_G(gc, obs, zs, zo, xs, ys, terms=terms)
                Go = oracle.closed_form_G(oc, obs, zs, zo, xs, ys, terms=terms)
                assert G.shape == (4, 3, 3, 3, 3)
                assert relerr(G, Go) < 1e-10, (src, obs, terms, relerr(G, Go))


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_green_1d_int8_tensor_cores_match_fp64(ytf, oracle, idx):
    """The 1D Bessel contraction on the int8 tensor cores (J_n(kρ) and the coefficient
    columns in three fixed-point digits, exact INT32 accumulation) against the FP64 path and
    the oracle, every source/obs layer and term selection: ≤ 1e-6 relative."""
    _, st = FOUNDATION_STACKS[idx]
    kx, wt = krho_grid(st, W, kmax=15.0)
    xs = np.array([-0.3, 0.0, 0.2, 0.45])
    ys = np.array([0.0, 0.15, -0.25])
    N = len(st)
    for src in range(1, N):
        gc = ytf.build_cavity_transfer_1d(st, W, src, kx, wt)
        zs = 0.4 * st[src - 1].d
        for obs in range(1, N + 1):
            d = st[obs - 1].d
            zo = [0.1 * d, 0.4 * d, 0.75 * d] if obs != src else [0.05 * d, 0.4 * d, 0.95 * d]
            for terms in (["all", "scattered", "toeplitz"] if obs == src else ["all"]):
                G64 = ytf.closed_form_G(gc, obs, zs, zo, xs, ys, terms=terms)
                G8 = ytf.closed_form_G(gc, obs, zs, zo, xs, ys, terms=terms, precision="int8x3")
                assert relerr(G8, G64) < 1e-6, (src, obs, terms, relerr(G8, G64))
    oc = oracle.build_cavity_transfer_1d(st, W, 1, kx, wt)
    gc = ytf.build_cavity_transfer_1d(st, W, 1, kx, wt)
    zo = [0.2 * st[0].d, 0.7 * st[0].d]
    assert relerr(ytf.closed_form_G(gc, 1, 0.4 * st[0].d, zo, xs, ys, precision="int8x3"),
                  oracle.closed_form_G(oc, 1, 0.4 * st[0].d, zo, xs, ys)) < 1e-6


def test_green_1d_int8_many_radii_nodes_and_rows(ytf):
    """The int8 Bessel contraction with several radius tiles (~300 distinct radii), node
    slices (40000 nodes) and column tiles (20 z rows: 200 order-0 columns > 160): ≤ 1e-6."""
    st = config1_stack()
    k0 = 2 * np.pi / 600.0
    panels = [(20 * k0 * i / 5000, 20 * k0 * (i + 1) / 5000) for i in range(5000)]
    kx, wt = ytf.gl_rule(panels, 8)
    gc = ytf.build_cavity_transfer_1d(st, k0, 1, kx, wt, obs_layers=[1])
    rho = np.geomspace(6.0, 3000.0, 300)
    zo = np.linspace(30.0, 190.0, 20)
    G64 = ytf.closed_form_G(gc, 1, 20.0, zo, rho, [0.0], terms="scattered")
    G8 = ytf.closed_form_G(gc, 1, 20.0, zo, rho, [0.0], terms="scattered", precision="int8x3")
    assert relerr(G8, G64) < 1e-6, relerr(G8, G64)
    assert relerr(G8[..., 2, 2], G64[..., 2, 2]) < 1e-6


def test_config1_gzz_1d_matches_oracle(ytf, oracle):
    """Vertical dipole 20 nm above the uniaxial film, real-axis GL panels to 20 k0."""
    st = config1_stack()
    k0 = 2 * np.pi / 600.0
    panels = [(20 * k0 * i / 128, 20 * k0 * (i + 1) / 128) for i in range(128)]
    kx, wt = oracle.gl_rule(panels, 8)
    gc = ytf.build_cavity_transfer_1d(st, k0, 1, kx, wt, obs_layers=[1])
    oc = oracle.build_cavity_transfer_1d(st, k0, 1, kx, wt, obs_layers=[1])
    rho = np.geomspace(6.0, 3000.0, 32)
    zo = np.linspace(0.0, 200.0, 9)
    zsrc = 20.0  # local height above the 1/2 interface
    G = ytf.closed_form_G(gc, 1, zsrc, zo, rho, [0.0])
    Go = oracle.closed_form_G(oc, 1, zsrc, zo, rho, [0.0])
    assert relerr(G[..., 2, 2], Go[..., 2, 2]) < 1e-10
    assert relerr(G, Go) < 1e-10


@pytest.mark.parametrize("idx", [3, 4])
def test_transfer_2d_full_solve_matches_oracle(ytf, oracle, idx):
    """Biaxial and gyrotropic stacks: the general 4x4 eigen path on the device."""
    _, st = FOUNDATION_STACKS[idx]
    kr, wr = krho_grid(st, W, kmax=10.0, width=1.0)
    ph, wp = uniform_phi(8)
    for src in (1, 2):
        gc = ytf.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp)
        oc = oracle.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp)
        _cmp_cache(gc, oc, tol=1e-8)
        xs = np.array([-0.2, 0.0, 0.3])
        for obs in range(1, len(st) + 1):
            d = st[obs - 1].d
            zo = [0.2 * d, 0.7 * d]
            G = ytf.closed_form_G(gc, obs, 0.3 * st[src - 1].d, zo, xs, xs)
            Go = oracle.closed_form_G(oc, obs, 0.3 * st[src - 1].d, zo, xs, xs)
            assert relerr(G, Go) < 1e-9, (src, obs, relerr(G, Go))


@pytest.mark.parametrize("nz", [3, 6, 8, 11])
def test_green_2d_even_rows_match_oracle(ytf, oracle, nz):
    """Evenly spaced z rows (the strength kernel steps the phases e^{i kz z} by recurrence
    where no row's exponent nears the clamp) on both sides of the source and in the other
    layers, with nodes far into the evanescent range (kρ up to 150 k0: exponents -Im(kz) z
    beyond 690, where the per-row clamped phase takes over): every precision agrees with the
    oracle as on unevenly spaced rows."""
    _, st = FOUNDATION_STACKS[4]
    kr, wr = krho_grid(st, W, kmax=150.0 * W, width=6.0)
    ph, wp = uniform_phi(6)
    src = 2
    gc = ytf.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp)
    oc = oracle.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp)
    xs = np.array([-0.2, 0.0, 0.3])
    zs = 0.45 * st[src - 1].d
    for obs in (src, 1, 3):
        d = st[obs - 1].d
        zo = np.linspace(0.05 * d, 0.95 * d, nz)
        Go = oracle.closed_form_G(oc, obs, zs, zo, xs, xs)
        assert relerr(ytf.closed_form_G(gc, obs, zs, zo, xs, xs), Go) < 1e-10, obs
        assert relerr(ytf.closed_form_G(gc, obs, zs, zo, xs, xs, precision="int8x3"), Go) < 1e-6, obs
        if obs == src:
            for terms in ("direct", "scattered", "toeplitz", "hankel"):
                Gt = ytf.closed_form_G(gc, obs, zs, zo, xs, xs, terms=terms)
                assert relerr(Gt, oracle.closed_form_G(oc, obs, zs, zo, xs, xs, terms=terms)) < 1e-10, terms


@pytest.mark.parametrize("shape", [(8, 6), (1, 5), (33, 2)])
def test_green_2d_int8_even_pixels_match_oracle(ytf, oracle, shape):
    """Evenly spaced pixel coordinates (the int8 path's phase tables are then stepped along each
    row by recurrence): int8x3 and split-BF16 G within 1e-6 of the oracle, like uneven pixels."""
    _, st = FOUNDATION_STACKS[3]
    kr, wr = krho_grid(st, W, kmax=12.0, width=1.0)
    ph, wp = uniform_phi(8)
    gc = ytf.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp, obs_layers=[2])
    oc = oracle.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp, obs_layers=[2])
    nx, ny = shape
    xs = np.linspace(-0.4, 0.35, nx) if nx > 1 else np.array([0.15])
    ys = np.linspace(0.3, -0.25, ny)
    d = st[1].d
    zo = [0.2 * d, 0.6 * d]
    Go = oracle.closed_form_G(oc, 2, 0.4 * d, zo, xs, ys)
    for prec in ("int8x3", "split_bf16"):
        G = ytf.closed_form_G(gc, 2, 0.4 * d, zo, xs, ys, precision=prec)
        assert relerr(G, Go) < 1e-6, (prec, relerr(G, Go))


def test_transfer_2d_rotation_fill_matches_oracle(ytf, oracle):
    st = [lay(m_vac, 1.0), lay(m_uni, 0.8), lay(m_gl, 0.5), lay(m_vac, 1.0)]
    kr, wr = krho_grid(st, W, kmax=12.0, width=1.0)
    ph, wp = uniform_phi(12)
    gc = ytf.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp)
    assert gc.rotation
    oc = oracle.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp)
    _cmp_cache(gc, oc)
    gf = ytf.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp, rotation=False)
    xs = np.array([-0.2, 0.1, 0.3])
    for obs in (1, 2, 3, 4):
        d = st[obs - 1].d
        G = ytf.closed_form_G(gc, obs, 0.35, [0.3 * d], xs, xs)
        assert relerr(G, oracle.closed_form_G(oc, obs, 0.35, [0.3 * d], xs, xs)) < 1e-10
        assert relerr(G, ytf.closed_form_G(gf, obs, 0.35, [0.3 * d], xs, xs)) < 1e-10


def test_free_space_dipole_on_gpu(ytf, oracle):
    """Absolute normalization on the device (Gz_ClosedForm_Point_Validation.jl [f])."""
    for omega in (2 * np.pi, 1.0):
        ef = 1.0 + 1e-4j
        st = [lay(IsotropicMaterial(ef), 3.0) for _ in range(3)]
        kx, wt, _ = oracle.fixed_grid_1d(st, omega, 2, h_min=0.025, rho_max=1.0, scan=False, rtol=1e-10)
        Gref = np.stack([e_free(np.array([0.4, 0, 0.7]), np.eye(3)[q].astype(complex), omega * np.sqrt(ef), ef)
                         for q in range(3)], axis=1)
        G1 = ytf.closed_form_G(ytf.build_cavity_transfer_1d(st, omega, 2, kx, wt), 2, 1.0, [1.7], [0.4], [0.0])[0, 0, 0]
        assert relerr(G1, Gref) < 1e-7


def test_gl_rule_bitexact_with_oracle(ytf, oracle):
    rng = np.random.default_rng(7)
    brk = np.sort(rng.uniform(0, 50, 40))
    panels = list(zip(brk[:-1], brk[1:]))
    sing = [brk[5], brk[17], brk[30]]
    for order in (8, 12):
        n, w = ytf.gl_rule(panels, order, sing)
        no, wo = oracle.gl_rule(panels, order, sing)
        assert np.array_equal(n, no) and np.array_equal(w, wo)


def test_argument_errors_match_reference_messages(ytf):
    st = [lay(m_vac, 1.0), lay(m_bi, 0.7), lay(m_vac, 1.0)]
    with pytest.raises(ytf.YTFError, match="source_layer=3 must be in 1:2"):
        ytf.build_cavity_transfer_1d(st, W, 3, [1.0], [1.0], check_symmetry=False)
    with pytest.raises(ytf.YTFError, match="requires an isotropic/uniaxial stack"):
        ytf.build_cavity_transfer_1d(st, W, 1, [1.0], [1.0])
    with pytest.raises(ytf.YTFError, match="rotation=true requires an azimuthally symmetric stack"):
        ytf.build_cavity_transfer_2d(st, W, 1, [1.0], [1.0], [0.0], [1.0], rotation=True)
    c = ytf.build_cavity_transfer_1d([lay(m_vac, 1.0), lay(m_gl, 0.7), lay(m_vac, 1.0)], W, 2, [1.0, 2.0], [0.5, 0.5],
                                     obs_layers=[2, 3])
    with pytest.raises(ytf.YTFError, match="not in this cache's obs_layers"):
        ytf.closed_form_G(c, 1, 0.3, [0.5], [0.0], [0.0])
    with pytest.raises(ytf.YTFError, match="terms needs obs_layer == source_layer"):
        ytf.closed_form_G(c, 3, 0.3, [0.5], [0.0], [0.0], terms="toeplitz")
    with pytest.raises(ytf.YTFError, match="outside"):
        ytf.closed_form_G(c, 2, 0.9, [0.5], [0.0], [0.0])


def test_empty_and_single_node_inputs(ytf, oracle):
    st = [lay(m_vac, 1.0), lay(m_gl, 0.7), lay(m_vac, 1.0)]
    c0 = ytf.build_cavity_transfer_1d(st, W, 2, [], [])
    G0 = ytf.closed_form_G(c0, 2, 0.3, [0.5], [0.1], [0.0])
    assert G0.shape == (1, 1, 1, 3, 3) and np.all(G0 == 0)
    c1 = ytf.build_cavity_transfer_1d(st, W, 2, [3.0], [0.25])
    o1 = oracle.build_cavity_transfer_1d(st, W, 2, [3.0], [0.25])
    assert relerr(ytf.closed_form_G(c1, 1, 0.3, [0.5], [0.1], [0.2]),
                  oracle.closed_form_G(o1, 1, 0.3, [0.5], [0.1], [0.2])) < 1e-12
    # ρ = 0 exactly and a ragged lateral grid
    xs = np.array([0.0, 0.05, 0.3]); ys = np.array([0.0])
    kx, wt = krho_grid(st, W, kmax=10.0)
    c = ytf.build_cavity_transfer_1d(st, W, 2, kx, wt)
    o = oracle.build_cavity_transfer_1d(st, W, 2, kx, wt)
    assert relerr(ytf.closed_form_G(c, 2, 0.3, [0.2, 0.5], xs, ys), oracle.closed_form_G(o, 2, 0.3, [0.2, 0.5], xs, ys)) < 1e-10


@pytest.mark.parametrize("prec", ["split_bf16", "int8x3"])
@pytest.mark.parametrize("idx", [3, 4])
def test_lateral_tensor_cores_match_fp64(ytf, oracle, idx, prec):
    """The tensor-core lateral synthesis against the FP64 path and the oracle: ≤ 1e-6
    relative (the metric's bound), on biaxial and gyrotropic stacks. split_bf16: 3-term
    BF16 split, FP32 accumulation in tensor memory; int8x3: three fixed-point base-256
    digits per operand, exact INT32 accumulation; both sum node slices in FP64."""
    _, st = FOUNDATION_STACKS[idx]
    kr, wr = krho_grid(st, W, kmax=10.0, width=0.5)
    ph, wp = uniform_phi(32)
    gc = ytf.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp, obs_layers=[1, 2, 3])
    xs = np.linspace(-0.3, 0.3, 11)
    ys = np.linspace(-0.25, 0.2, 9)
    for obs, zo in ((2, [0.1, 0.35, 0.6]), (1, [0.4]), (3, [0.2, 0.3])):
        G64 = ytf.closed_form_G(gc, obs, 0.3, zo, xs, ys)
        Gtc = ytf.closed_form_G(gc, obs, 0.3, zo, xs, ys, precision=prec)
        assert relerr(Gtc, G64) < 1e-6, (obs, relerr(Gtc, G64))
    oc = oracle.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp, obs_layers=[2])
    Go = oracle.closed_form_G(oc, 2, 0.3, [0.1, 0.6], xs, ys)
    assert relerr(ytf.closed_form_G(gc, 2, 0.3, [0.1, 0.6], xs, ys, precision=prec), Go) < 1e-6


@pytest.mark.parametrize("prec", ["split_bf16", "int8x3"])
def test_lateral_tensor_cores_ragged_tiles(ytf, prec):
    """Pixel counts and column counts that do not fill a 128-pixel tile or a 16-wide MMA,
    node counts that do not fill a 16-node stage, and more than 128 columns (two N-tiles)."""
    _, st = FOUNDATION_STACKS[4]
    kr, wr = krho_grid(st, W, kmax=6.0, width=0.7)
    ph, wp = uniform_phi(6)
    gc = ytf.build_cavity_transfer_2d(st, W, 2, kr[:-3], wr[:-3], ph, wp, obs_layers=[2])
    for nx, ny, nz in ((1, 1, 1), (7, 3, 2), (13, 11, 16)):
        xs = np.linspace(-0.2, 0.3, nx)
        ys = np.linspace(-0.1, 0.15, ny)
        zo = list(np.linspace(0.05, 0.85, nz))
        G64 = ytf.closed_form_G(gc, 2, 0.3, zo, xs, ys)
        Gtc = ytf.closed_form_G(gc, 2, 0.3, zo, xs, ys, precision=prec)
        assert relerr(Gtc, G64) < 1e-6, (nx, ny, nz, relerr(Gtc, G64))


def test_lateral_int8_slices_capped_and_exact(ytf):
    """int8x3 with more pixel tiles than SMs, so one CTA would take every node: the host
    caps a node slice at 16384 nodes (INT32 headroom) and the slices are summed in FP64.
    The integer contraction is exact, so two calls agree bit for bit. The error, ~1.5e-7
    here (a numpy restatement of the digit scheme gives the same figure), is dominated by
    the dropped weight-256 digit products; the phase digits alone contribute ~6e-9."""
    _, st = FOUNDATION_STACKS[3]
    kr, wr = krho_grid(st, W, kmax=8.0, width=0.5)
    nphi = max(1, -(-20000 // len(kr)))
    ph, wp = uniform_phi(nphi)
    gc = ytf.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp, obs_layers=[2])
    assert gc.n > 16384
    xs = np.linspace(-0.3, 0.3, 160)
    ys = np.linspace(-0.25, 0.2, 120)
    G64 = ytf.closed_form_G(gc, 2, 0.3, [0.45], xs, ys)
    G8 = ytf.closed_form_G(gc, 2, 0.3, [0.45], xs, ys, precision="int8x3")
    assert relerr(G8, G64) < 3e-7, relerr(G8, G64)
    assert np.array_equal(G8, ytf.closed_form_G(gc, 2, 0.3, [0.45], xs, ys, precision="int8x3"))


def _exports_equal(a, b):
    ea, eb = a.export(), b.export()
    for key in ea:
        assert np.array_equal(np.asarray(ea[key]), np.asarray(eb[key])), key
    for x, y in zip(a.status(), b.status()):
        assert np.array_equal(x, y)


def test_transfer_batch_matches_single_builds(ytf):
    """One ytf_transfer_batch call over a mixed, uneven batch (1D and 2D, forward-only and
    general chains, different stacks, layer counts, sizes and frequencies, a rotation item
    and an empty rule) returns, item by item, the caches of the single builds bit for bit:
    the batched kernels run the same per-node code on each item's own parameters."""
    items, singles = [], []
    for idx, src, obs, nk in ((0, 1, None, 48), (1, 2, [2], 100), (2, 1, [1, 3], 7), (2, 2, [2], 0)):
        _, st = FOUNDATION_STACKS[idx]
        kx, wt = krho_grid(st, W * (1 + 0.1 * idx), kmax=12.0)
        kx, wt = kx[:nk], wt[:nk]
        items.append(dict(stack=st, omega=W * (1 + 0.1 * idx), source_layer=src, kx_nodes=kx, wt_nodes=wt,
                          obs_layers=obs))
        singles.append(ytf.build_cavity_transfer_1d(st, W * (1 + 0.1 * idx), src, kx, wt, obs_layers=obs))
    for idx, src, obs, nphi, rot in ((3, 2, [2], 5, "auto"), (4, 1, None, 3, "auto"), (4, 2, [2], 8, "auto"),
                                     (1, 2, [2, 3], 4, "auto"), (1, 2, [2], 4, False)):
        _, st = FOUNDATION_STACKS[idx]
        kr, wr = krho_grid(st, W, kmax=10.0)
        ph, wp = uniform_phi(nphi)
        items.append(dict(stack=st, omega=W, source_layer=src, kr_nodes=kr, kr_weights=wr, phi_nodes=ph,
                          phi_weights=wp, obs_layers=obs, rotation=rot))
        singles.append(ytf.build_cavity_transfer_2d(st, W, src, kr, wr, ph, wp, obs_layers=obs, rotation=rot))
    batch = ytf.build_cavity_transfer_batch(items)
    assert len(batch) == len(singles)
    assert batch[-2].rotation and not batch[-1].rotation
    for b, s in zip(batch, singles):
        assert b.n == s.n and b.obs_layers == s.obs_layers
        _exports_equal(b, s)


def test_transfer_batch_argument_error_names_the_item(ytf):
    _, st = FOUNDATION_STACKS[1]
    kx, wt = krho_grid(st, W, kmax=5.0)
    good = dict(stack=st, omega=W, source_layer=1, kx_nodes=kx, wt_nodes=wt)
    bad = dict(good, source_layer=len(st))
    with pytest.raises(ytf.YTFError, match=r"source_layer=.*batch item 1"):
        ytf.build_cavity_transfer_batch([good, bad])


def test_green_batch_matches_single_calls(ytf):
    """ytf_green_batch over 1D and 2D caches, every precision, host and device outputs:
    item for item the same arrays as closed_form_G (bit for bit)."""
    import torch
    _, st1 = FOUNDATION_STACKS[1]
    kx, wt = krho_grid(st1, W, kmax=12.0)
    c1 = ytf.build_cavity_transfer_1d(st1, W, 2, kx, wt)
    _, st4 = FOUNDATION_STACKS[4]
    kr, wr = krho_grid(st4, W, kmax=10.0)
    ph, wp = uniform_phi(6)
    c2 = ytf.build_cavity_transfer_2d(st4, W, 2, kr, wr, ph, wp, obs_layers=[2])
    xs, ys = np.linspace(-0.3, 0.3, 9), np.linspace(-0.2, 0.25, 7)
    specs = [(c1, 2, 0.3, [0.1, 0.4], xs, ys, "fp64"), (c2, 2, 0.3, [0.2], xs, ys, "int8x3"),
             (c2, 2, 0.3, [0.2, 0.6], xs[:5], ys, "split_bf16"), (c2, 2, 0.3, [0.5], xs, ys[:3], "fp64"),
             (c2, 2, 0.3, [0.5], xs, ys, "int8x3")]
    dev = torch.empty(len(xs) * len(ys) * 9, dtype=torch.complex128, device="cuda")
    items = [dict(cache=c, obs_layer=o, zsrc_local=z, z_obs=zo, xs=x, ys=y, precision=p)
             for c, o, z, zo, x, y, p in specs]
    items[-1]["out"] = dev
    res = ytf.closed_form_G_batch(items)
    for (c, o, z, zo, x, y, p), r in zip(specs, res):
        ref = ytf.closed_form_G(c, o, z, zo, x, y, precision=p)
        got = r.cpu().numpy().reshape(3, 3, 1, len(y), len(x)).transpose(4, 3, 2, 1, 0) if hasattr(r, "cpu") else r
        assert np.array_equal(got, ref), p


def test_green_batch_all_1d_side_streams_match_single_calls(ytf):
    """An all-1D ytf_green_batch (FP64 and contour items round-robin on side streams with
    their own workspaces, radii maps pre-uploaded; int8x3 items in the grouped synthesis):
    item for item the same arrays as closed_form_G, bit for bit for FP64 and the contour, to
    the int8x3 tolerance for the grouped items (their node slices differ), for several stacks,
    node counts, repeated radii, host and device outputs."""
    import torch
    specs, caches = [], []
    for idx, kmax, src in ((1, 12.0, 2), (0, 6.0, 1), (2, 9.0, 1), (1, 4.0, 1)):
        _, st = FOUNDATION_STACKS[idx]
        kx, wt = krho_grid(st, W, kmax=kmax)
        caches.append(ytf.build_cavity_transfer_1d(st, W, src, kx, wt, obs_layers=[src]))
    _, stc = FOUNDATION_STACKS[1]
    kc, wc = ytf.contour_rule(W, npanels=64)
    caches.append(ytf.build_cavity_transfer_1d_contour(stc, W, 1, kc, wc, obs_layers=[1]))
    xs, ys = np.linspace(-0.3, 0.3, 9), np.linspace(-0.2, 0.25, 7)
    rho = np.geomspace(0.01, 2.0, 40)
    for j, c in enumerate(caches):
        src = c.source_layer
        for prec in (("fp64", "int8x3") if j < 4 else ("fp64",)):
            specs.append((c, src, 0.3, [0.1, 0.4, 0.7], rho, [0.0], prec))
            specs.append((c, src, 0.3, [0.2], xs, ys, prec))
    items = [dict(cache=c, obs_layer=o, zsrc_local=z, z_obs=zo, xs=x, ys=y, precision=p)
             for c, o, z, zo, x, y, p in specs]
    for i in (1, 4, 7):
        x, y, zo = items[i]["xs"], items[i]["ys"], items[i]["z_obs"]
        items[i]["out"] = torch.empty(len(x) * len(y) * len(zo) * 9, dtype=torch.complex128, device="cuda")
    for rep in range(2):  # the second pass reuses the slots' workspaces
        res = ytf.closed_form_G_batch(items)
        for (c, o, z, zo, x, y, p), r in zip(specs, res):
            ref = ytf.closed_form_G(c, o, z, zo, x, y, precision=p)
            if hasattr(r, "cpu"):
                r = r.cpu().numpy().reshape(3, 3, len(zo), len(y), len(x)).transpose(4, 3, 2, 1, 0)
            if p == "int8x3":
                assert relerr(r, ref) < 1e-6, (p, len(x), len(y), relerr(r, ref))
            else:
                assert np.array_equal(r, ref), (p, len(x), len(y))


def test_grouped_1d_int8_synthesis(ytf):
    """The grouped 1D int8x3 synthesis of ytf_green_batch: 40 items of four stacks, rules of
    8 to ~2000 nodes (node counts off the 64-node stage), one to five heights, radii lists
    and 2D pixel grids with repeated radii, host and device outputs, with FP64, 2D and
    deformed-contour items between them (those take the per-item path). Every grouped item's
    G matches the FP64 synthesis to 1e-6 (or to twice the per-item int8x3 path's own error,
    where that is larger); with a 2 MB group bound (one or two items per
    group) the results are bit for bit those of the default bound (one group); and a second
    pass reuses the workspace."""
    import torch
    ctx = ytf.default_context()
    rng = np.random.default_rng(5)
    caches = []
    for idx, kmax, src in ((1, 12.0, 2), (0, 6.0, 1), (2, 9.0, 1), (1, 4.0, 1), (2, 8.0, 2)):
        _, st = FOUNDATION_STACKS[idx]
        kx, wt = krho_grid(st, W, kmax=kmax)
        caches.append(ytf.build_cavity_transfer_1d(st, W, src, kx, wt, obs_layers=[src]))
        caches.append(ytf.build_cavity_transfer_1d(st, W, src, kx[:8], wt[:8], obs_layers=[src]))
        caches.append(ytf.build_cavity_transfer_1d(st, W, src, kx[:1000:3], wt[:1000:3], obs_layers=[src]))
    _, stc = FOUNDATION_STACKS[1]
    kc, wc = ytf.contour_rule(W, npanels=32)
    cc = ytf.build_cavity_transfer_1d_contour(stc, W, 1, kc, wc, obs_layers=[1])
    _, st2 = FOUNDATION_STACKS[4]
    kr2, wr2 = krho_grid(st2, W, kmax=6.0)
    ph, wp = uniform_phi(4)
    c2 = ytf.build_cavity_transfer_2d(st2, W, 2, kr2, wr2, ph, wp, obs_layers=[2])
    xs, ys = np.linspace(-0.3, 0.3, 7), np.linspace(-0.2, 0.25, 5)
    specs = []
    for j in range(40):
        c = caches[j % len(caches)]
        nz = 1 + j % 5
        zo = list(np.sort(rng.uniform(0.05, 0.9, nz)))
        if j % 3 == 0:
            x, y = xs, ys
        else:
            x, y = np.geomspace(0.01, 2.0, 20 + 7 * (j % 4)), [0.0]
        specs.append(dict(cache=c, obs_layer=c.source_layer, zsrc_local=0.3, z_obs=zo, xs=x, ys=y,
                          precision="int8x3", terms=("all", "scattered")[j % 2]))
        if j % 7 == 3:
            specs.append(dict(cache=cc, obs_layer=1, zsrc_local=0.3, z_obs=[0.2], xs=x, ys=y, precision="fp64"))
        if j % 11 == 5:
            specs.append(dict(cache=c2, obs_layer=2, zsrc_local=0.3, z_obs=[0.4], xs=xs, ys=ys, precision="int8x3"))
        if j % 9 == 2:
            specs.append(dict(specs[-1], precision="fp64"))

    def run(group_bytes):
        ctx.set_group_bytes(group_bytes)
        items = []
        for k, it in enumerate(specs):
            it = dict(it)
            if k % 4 == 1:
                it["out"] = torch.empty(len(it["xs"]) * len(it["ys"]) * len(it["z_obs"]) * 9, dtype=torch.complex128,
                                        device="cuda")
            items.append(it)
        res = ytf.closed_form_G_batch(items)
        out = []
        for it, r in zip(items, res):
            if hasattr(r, "cpu"):
                r = r.cpu().numpy().reshape(3, 3, len(it["z_obs"]), len(it["ys"]), len(it["xs"])).transpose(4, 3, 2, 1, 0)
            out.append(r)
        return out

    try:
        big = run(0)
        small = run(2 << 20)
        again = run(2 << 20)
    finally:
        ctx.set_group_bytes(0)
    for it, a, b, c in zip(specs, big, small, again):
        assert np.array_equal(a, b) and np.array_equal(b, c), it["precision"]
        kw = {k: it[k] for k in ("z_obs", "xs", "ys", "terms") if k in it}
        ref = ytf.closed_form_G(it["cache"], it["obs_layer"], it["zsrc_local"], precision="fp64", **kw)
        if it["precision"] == "int8x3" and not it["cache"].is2d:
            # the per-item int8x3 path on the same item bounds what the digits can resolve
            # (rules of 8 nodes integrate to little next to their terms)
            e_single = relerr(ytf.closed_form_G(it["cache"], it["obs_layer"], it["zsrc_local"], precision="int8x3", **kw),
                              ref)
            assert relerr(a, ref) <= max(1e-6, 2 * e_single), (relerr(a, ref), e_single, it["cache"].n)
        else:
            single = ytf.closed_form_G(it["cache"], it["obs_layer"], it["zsrc_local"], precision=it["precision"], **kw)
            assert np.array_equal(a, single)


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_cavity_response_matches_oracle(ytf, oracle, idx):
    """_cavity_response on the device (forward-only chain in response mode) against the
    oracle, every source layer, across the light lines and the guided-mode region."""
    _, st = FOUNDATION_STACKS[idx]
    ks = np.linspace(0.05, 4.0, 97) * W
    for src in range(1, len(st)):
        g = ytf.cavity_response(st, W, src, ks)
        o = np.array([oracle.cavity_response(st, W, src, k) for k in ks])
        assert relerr(g, o) < 1e-9, (src, relerr(g, o))


def test_point_kx_grid_without_scan_bit_exact(ytf, oracle):
    """point_kx_grid with the pole scan off: light lines, panels (host) and Gauss–Legendre
    nodes (device) equal the oracle's rule bit for bit."""
    for idx in (0, 1, 2):
        _, st = FOUNDATION_STACKS[idx]
        for h, rho in ((0.05, 1.0), (0.2, 0.0)):
            k, w, info = ytf.point_kx_grid(st, W, 1, h_min=h, rho_max=rho, scan=False)
            ko, wo, io = oracle.fixed_grid_1d(st, W, 1, h_min=h, rho_max=rho, scan=False)
            assert np.array_equal(k, ko) and np.array_equal(w, wo), idx
            assert info["Kcut"] == io["Kcut"] and info["n_panels"] == io["n_panels"]


def test_point_kx_grid_with_pole_scan_matches_oracle(ytf, oracle):
    """With the real-axis pole scan (device cavity responses, host peak search): the same
    poles and panels as the oracle's scan to refinement precision, and G integrated with
    either rule agrees to 1e-9."""
    from helpers import config1_like_stack
    for st, src in ((FOUNDATION_STACKS[1][1], 2), (config1_like_stack(), 1)):
        k, w, info = ytf.point_kx_grid(st, W, src, h_min=0.05, rho_max=1.0)
        ko, wo, io = oracle.fixed_grid_1d(st, W, src, h_min=0.05, rho_max=1.0)
        assert info["n_poles"] == io["n_poles"] and info["n_panels"] == io["n_panels"]
        assert len(k) == len(ko)
        assert np.max(np.abs(k - ko)) <= 1e-9 * info["Kcut"]
        c = ytf.build_cavity_transfer_1d(st, W, src, k, w, obs_layers=[src])
        co = ytf.build_cavity_transfer_1d(st, W, src, ko, wo, obs_layers=[src])
        xs, ys = np.array([0.1, 0.4]), np.array([0.0, 0.3])
        d = st[src - 1].d
        G = ytf.closed_form_G(c, src, 0.3 * d, [0.6 * d], xs, ys)
        Go = ytf.closed_form_G(co, src, 0.3 * d, [0.6 * d], xs, ys)
        assert relerr(G, Go) < 1e-9


def test_uneven_batch_workload_shape(ytf, oracle):
    """The uneven-batch workload at reduced node counts: 24 stacks of 2-24 layers (isotropic,
    uniaxial-hyperbolic, gyrotropic; 1D and 2D rules) built in one ytf_transfer_batch call
    equal the single builds bit for bit, and the smallest items match the oracle."""
    import bench
    tr, syn = bench.uneven_batch(n_stacks=24, nk_lo=64, nk_hi=512)
    assert len({len(t["stack"]) for t in tr}) > 5
    batch = ytf.build_cavity_transfer_batch(tr)
    for t, b in zip(tr, batch):
        if "kx_nodes" in t:
            s = ytf.build_cavity_transfer_1d(t["stack"], t["omega"], t["source_layer"], t["kx_nodes"], t["wt_nodes"],
                                             obs_layers=t["obs_layers"])
        else:
            s = ytf.build_cavity_transfer_2d(t["stack"], t["omega"], t["source_layer"], t["kr_nodes"], t["kr_weights"],
                                             t["phi_nodes"], t["phi_weights"], obs_layers=t["obs_layers"], rotation=False)
        _exports_equal(b, s)
    order = sorted(range(len(tr)), key=lambda i: len(tr[i].get("kx_nodes", ())) or 8 * len(tr[i]["kr_nodes"]))
    for i in order[:3]:
        t, y = tr[i], syn[i]
        if "kx_nodes" in t:
            oc = oracle.build_cavity_transfer_1d(t["stack"], t["omega"], t["source_layer"], t["kx_nodes"], t["wt_nodes"],
                                                 obs_layers=t["obs_layers"])
        else:
            oc = oracle.build_cavity_transfer_2d(t["stack"], t["omega"], t["source_layer"], t["kr_nodes"],
                                                 t["kr_weights"], t["phi_nodes"], t["phi_weights"],
                                                 obs_layers=t["obs_layers"], rotation=False)
        G = ytf.closed_form_G_batch([dict(y, cache=batch[i])])[0]
        Go = oracle.closed_form_G(oc, y["obs_layer"], y["zsrc_local"], y["z_obs"], y["xs"], y["ys"])
        assert relerr(G, Go) < 1e-9, (i, relerr(G, Go))


def test_complex_bessel_matches_mpmath(ytf):
    """J_0, J_1, J_2 of complex argument on the device (series, Miller recurrence, Hankel
    expansion) against mpmath, |z| up to 700, -2 <= Im z <= 0.5: within 1e-12 of the
    envelope sqrt(2/(π|z|)) e^{|Im z|} (1 below |z| = 1)."""
    import mpmath
    rng = np.random.default_rng(5)
    r = np.exp(rng.uniform(np.log(1e-3), np.log(700.0), 400))
    z = r * np.exp(1j * rng.uniform(-0.003, 0.0, 400)) + 1j * rng.uniform(-2.0, 0.5, 400)
    z = np.concatenate([z, [8.0 - 0.1j, 8.0001 + 0.0j, 24.999 - 1.0j, 25.0, 1.0 - 0.5j, 0.999j * 0 + 0.999]])
    env = np.where(np.abs(z) > 1, np.sqrt(2 / (np.pi * np.abs(z))) * np.exp(np.abs(z.imag)), np.exp(np.abs(z.imag)))
    for n in (0, 1, 2):
        g = ytf.bessel_j(n, z)
        ref = np.array([complex(mpmath.besselj(n, complex(v))) for v in z])
        err = np.abs(g - ref) / env
        assert np.max(err) < 1e-12, (n, np.max(err), z[np.argmax(err)])


def test_contour_with_zero_indentation_equals_real_axis_path(ytf):
    """The complex-node path with zero imaginary parts reproduces the real-node path."""
    st = config1_stack()
    k0 = 2 * np.pi / 600.0
    k, w = ytf.contour_rule(k0, npanels=64, h=0.0)
    gc = ytf.build_cavity_transfer_1d_contour(st, k0, 1, k, w, obs_layers=[1])
    gr = ytf.build_cavity_transfer_1d(st, k0, 1, k.real, w.real, obs_layers=[1])
    rho = np.geomspace(6.0, 3000.0, 12)
    zo = np.linspace(30.0, 190.0, 5)
    Gc = ytf.closed_form_G(gc, 1, 20.0, zo, rho, [0.0])
    Gr = ytf.closed_form_G(gr, 1, 20.0, zo, rho, [0.0])
    assert relerr(Gc, Gr) < 1e-13, relerr(Gc, Gr)


def test_config1_contour_matches_real_axis_oracle(ytf, oracle):
    """The 3-layer dipole problem at its full size: vertical dipole 20 nm above the uniaxial
    film, 4096 nodes (512 GL-8 panels) on the contour kρ = t - 0.05 i k0 sin(π t / 20 k0),
    t in [0, 20 k0], G on 256 radii log-spaced over 6-3000 nm x 64 heights over 0-200 nm. With
    the film's loss every pole lies above the real axis and the branch points on it, so by
    Cauchy's theorem the contour integral equals the oracle's real-axis integral over
    [0, 20 k0] (dense rule: breaks at the light lines, u² substitution at the half-space
    ones, ~48k nodes): G and Gzz within 1e-6 (FP64 contraction; the int8x3 one within 1e-6
    of it)."""
    st = config1_stack()
    k0 = 2 * np.pi / 600.0
    oracle.set_threads(__import__("os").cpu_count() or 1)
    k, w = ytf.contour_rule(k0, npanels=512, order=8)
    gc = ytf.build_cavity_transfer_1d_contour(st, k0, 1, k, w, obs_layers=[1])
    rho = np.geomspace(6.0, 3000.0, 256)
    zo = np.linspace(0.0, 200.0, 64)
    Gc = ytf.closed_form_G(gc, 1, 20.0, zo, rho, [0.0])
    lines = sorted({float(x) for L in st for x in oracle.light_lines(L, k0, 0.0) if 0 < x < 20 * k0})
    sing = sorted({float(x) for L in (st[0], st[-1]) for x in oracle.light_lines(L, k0, 0.0)})
    brk = [0.0] + lines + [20 * k0]
    panels = []
    for a, b in zip(brk[:-1], brk[1:]):
        n = max(8, int(np.ceil(6000 * (b - a) / (20 * k0))))
        e = np.linspace(a, b, n + 1)
        panels += list(zip(e[:-1], e[1:]))
    kr, wr = oracle.gl_rule(panels, 8, singular=sing)
    oc = oracle.build_cavity_transfer_1d(st, k0, 1, kr, wr, obs_layers=[1])
    Go = oracle.closed_form_G(oc, 1, 20.0, zo, rho, [0.0])
    assert relerr(Gc, Go) < 1e-6, relerr(Gc, Go)
    assert relerr(Gc[..., 2, 2], Go[..., 2, 2]) < 1e-6
    # the int8 tensor-core contraction on the contour (complex J_n as real and imaginary digit
    # images, two int8x3 contractions per order): within 1e-6 of the FP64 contour G, and so of
    # the oracle's real-axis integral
    G8 = ytf.closed_form_G(gc, 1, 20.0, zo, rho, [0.0], precision="int8x3")
    assert relerr(G8, Gc) < 1e-6, relerr(G8, Gc)
    assert relerr(G8, Go) < 1.5e-6, relerr(G8, Go)
    assert relerr(G8[..., 2, 2], Go[..., 2, 2]) < 1.5e-6


def test_point_krho_grid_2d_without_scan_bit_exact(ytf, oracle):
    """point_kρ_grid_2d with the pole scan off: the scanned directions' light lines, the
    panels and N_φ (host) and the Gauss–Legendre nodes (device) equal the oracle's bit for bit,
    for an azimuthally symmetric, a diagonal (biaxial) and a non-diagonal (gyrotropic) stack."""
    for idx in (2, 3, 4):
        _, st = FOUNDATION_STACKS[idx]
        for h, rho in ((0.05, 1.0), (0.2, 0.0)):
            k, w, ph, wp, info = ytf.point_krho_grid_2d(st, W, 2, h_min=h, rho_max=rho, scan=False)
            ko, wo, io = oracle.fixed_grid_2d(st, W, 2, h_min=h, rho_max=rho, scan=False)
            assert np.array_equal(k, ko) and np.array_equal(w, wo), idx
            assert info["Kcut"] == io["Kcut"] and info["n_panels"] == io["n_panels"]
            assert info["N_phi"] == io["N_phi"] and len(ph) == io["N_phi"] and np.allclose(wp.sum(), 2 * np.pi)


def test_point_krho_grid_2d_with_pole_scan_matches_oracle(ytf, oracle):
    """With the pole scan along every scanned direction (device cavity responses, host peak
    search): the same poles, panels and N_φ (the pole-track term included) as the oracle's
    scan to refinement precision -- a golden-section maximum is fixed only to about √eps of
    its position (the response is flat to rounding within that), so the device's and the
    host's rounding move node positions by up to ~1e-8 Kcut -- and G on a (kρ, φ) grid built
    from either rule agrees to 1e-9."""
    for idx, n_scan in ((3, 8), (4, 8)):
        _, st = FOUNDATION_STACKS[idx]
        k, w, ph, wp, info = ytf.point_krho_grid_2d(st, W, 2, h_min=0.1, rho_max=0.5, N_phi_scan=n_scan)
        ko, wo, io = oracle.fixed_grid_2d(st, W, 2, h_min=0.1, rho_max=0.5, n_phi_scan=n_scan)
        assert info["n_poles"] == io["n_poles"] and info["n_panels"] == io["n_panels"], idx
        assert len(k) == len(ko) and np.max(np.abs(k - ko)) <= 1e-7 * info["Kcut"]
        assert abs(info["N_phi"] - io["N_phi"]) <= max(2, 1e-6 * io["N_phi"])
        phs, wps = uniform_phi(16)
        c = ytf.build_cavity_transfer_2d(st, W, 2, k, w, phs, wps, obs_layers=[2])
        co = ytf.build_cavity_transfer_2d(st, W, 2, ko, wo, phs, wps, obs_layers=[2])
        xs = np.array([0.1, 0.4])
        d = st[1].d
        G = ytf.closed_form_G(c, 2, 0.3 * d, [0.6 * d], xs, xs)
        Go = ytf.closed_form_G(co, 2, 0.3 * d, [0.6 * d], xs, xs)
        assert relerr(G, Go) < 1e-9


def test_adaptive_seeds_match_oracle(ytf, oracle):
    """adaptive_seeds on the features of a point rule: bit for bit without the pole scan; with
    it, the same seeds to the scan's refinement precision."""
    for idx in (0, 1, 2):
        _, st = FOUNDATION_STACKS[idx]
        s = ytf.adaptive_seeds(st, W, 2 if len(st) > 2 else 1, h_min=0.05, rho_max=1.0, scan=False)
        so = oracle.adaptive_seeds(st, W, 2 if len(st) > 2 else 1, h_min=0.05, rho_max=1.0, scan=False)
        assert np.array_equal(s, so), idx
    _, st = FOUNDATION_STACKS[1]
    s = ytf.adaptive_seeds(st, W, 2, h_min=0.05, rho_max=1.0)
    so = oracle.adaptive_seeds(st, W, 2, h_min=0.05, rho_max=1.0)
    assert len(s) == len(so) and np.max(np.abs(s - so)) <= 1e-9 * so[-1]


def test_1d_synthesis_in_node_passes_equals_the_sum_of_its_parts(ytf):
    """A 1D rule larger than one synthesis pass (262144 nodes) is synthesised in passes whose
    P_n are summed: G on the whole rule equals the sum of G on two halves of it (each one
    pass) to rounding in FP64, and the int8x3 form agrees with FP64 to its tolerance."""
    from helpers import config1_like_stack
    st = config1_like_stack()
    n = 300_000
    e = np.linspace(0.0, 30.0 * W, n // 8 + 1)
    x, wg = np.polynomial.legendre.leggauss(8)
    k = (0.5 * (e[1:] + e[:-1])[:, None] + 0.5 * np.diff(e)[:, None] * x[None, :]).ravel()
    w = (0.5 * np.diff(e)[:, None] * wg[None, :]).ravel()
    zo, rho = [0.05, 0.2], np.geomspace(0.02, 3.0, 16)
    G = lambda kk, ww, p="fp64": ytf.closed_form_G(ytf.build_cavity_transfer_1d(st, W, 1, kk, ww, obs_layers=[1]), 1,
                                                   0.03, zo, rho, [0.0], terms="scattered", precision=p)
    whole = G(k, w)
    h = n // 2
    parts = G(k[:h], w[:h]) + G(k[h:], w[h:])
    assert relerr(whole, parts) < 1e-12
    assert relerr(G(k, w, "int8x3"), whole) < 1e-6


def test_real_bessel_pair_of_the_int8_synthesis(ytf):
    """ytf_bessel_j01: J_0, J_1 of real arguments as the int8x3 J images take them (the CUDA
    library below 25, Hankel's asymptotic pair with a shared phase above) against scipy, to
    2e-12 absolute over 0-8000 (dense around the switch at 25), odd/even symmetry for x < 0."""
    from scipy.special import j0, j1
    x = np.concatenate([np.linspace(0.0, 40.0, 40001), np.linspace(24.9, 25.1, 2001), np.geomspace(40.0, 8000.0, 200001)])
    a, b = ytf.bessel_j01(x)
    assert np.max(np.abs(a - j0(x))) < 2e-12
    assert np.max(np.abs(b - j1(x))) < 2e-12
    an, bn = ytf.bessel_j01(-x)
    assert np.max(np.abs(an - a)) < 1e-15 and np.max(np.abs(bn + b)) < 1e-15
