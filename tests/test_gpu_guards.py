"""The numerical guards and failure paths of the solve, through the C ABI, against the oracle.

* A singular interface (two identical vacuum layers met at tangential incidence, kx = ω: both
  forward modes coincide, so the interface matrix [-Vf_B Vb_A] has rank 2 and the LU meets an
  exact zero pivot) takes the reference's pivoted-QR least-squares branch
  (mod_ScatteringMatrix.jl:35-44); the node stays valid.
* Non-finite or ε33 = 0 materials: a closed-form layer (isotropic/uniaxial) makes its nodes'
  T^o non-finite, so Tvalid is false and only the direct term survives, as in the reference
  (mod_CavityTransfer.jl:226-251); a general-path layer makes Julia's eigen raise
  "matrix contains Infs or NaNs", which the reference's per-node catch does not catch, so the
  whole build fails.
* The bounded waits of the int8 tensor-core pipelines: with the poll limit at 1 they run
  out, the call returns an error instead of a result, and the context stays usable.
"""
import numpy as np
import pytest

from helpers import krho_grid, relerr, uniform_phi
from yellowthinfilms_b200.materials import BiaxialMaterial, FlatOpticalLayer, IsotropicMaterial, UniaxialMaterial

pytestmark = pytest.mark.gpu

W = 2 * np.pi
lay = FlatOpticalLayer


def _caches(api, oracle, st, k, w, obs):
    return (api.build_cavity_transfer_1d(st, W, 1, k, w, obs_layers=obs),
            oracle.build_cavity_transfer_1d(st, W, 1, k, w, obs_layers=obs))


@pytest.mark.parametrize("obs", [[1], [1, 2, 3]])
def test_singular_interface_takes_the_pivoted_qr_branch(oracle, obs):
    """obs [1]: the forward-only chain (interfaces on raw mode columns); obs [1, 2, 3]: the
    general chain. The tangential node's cache and G match the oracle's QR branch."""
    from yellowthinfilms_b200 import api
    st = [lay(IsotropicMaterial(2.25), 0.5), lay(IsotropicMaterial(1.0), 0.3), lay(IsotropicMaterial(1.0), 0.4),
          lay(IsotropicMaterial(2.25), 0.5)]
    k = np.array([0.5 * W, W, 1.2 * W, 1.4 * W])
    w = np.full(4, 0.05)
    g, o = _caches(api, oracle, st, k, w, obs)
    valid, tvalid, status = g.status()
    eo = o.export()
    assert valid.all() and np.array_equal(valid, eo["valid"].astype(bool))
    assert np.array_equal(tvalid, np.asarray(eo["Tvalid"]).reshape(tvalid.shape).astype(bool))
    assert not (status & 8).any()  # no singular flag: the QR branch solved the interface
    eg = g.export()
    assert relerr(eg["T"], eo["T"]) < 1e-10
    for key in ("sf", "sb", "Qf", "Qb"):
        assert relerr(eg[key], eo[key]) < 1e-10, key
    zo, xs = [0.1, 0.3], [0.05, 0.2, 0.6]
    assert relerr(api.closed_form_G(g, 1, 0.2, zo, xs, [0.0]), oracle.closed_form_G(o, 1, 0.2, zo, xs, [0.0])) < 1e-10


@pytest.mark.parametrize("bad", [IsotropicMaterial(complex(np.nan, 0.0)), UniaxialMaterial(2.0 + 0.1j, 0.0),
                                 IsotropicMaterial(complex(np.inf, 0.0))], ids=["nan", "eps33=0", "inf"])
def test_non_finite_closed_form_layer_clears_Tvalid(oracle, bad):
    """A non-finite closed-form layer below the source: every node's T^o is non-finite, so
    Tvalid is false (status bit 32) while the source seeds stay valid; G is the direct term
    alone, equal to the oracle's."""
    import warnings
    from yellowthinfilms_b200 import api
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        st = [lay(IsotropicMaterial(1.0), 0.5), lay(bad, 0.3), lay(IsotropicMaterial(2.25), 0.5)]
    k = np.linspace(0.1, 3.0, 6) * W
    w = np.full(6, 0.1)
    g, o = _caches(api, oracle, st, k, w, [1])
    valid, tvalid, status = g.status()
    eo = o.export()
    assert np.array_equal(valid, eo["valid"].astype(bool)) and valid.all()
    assert not tvalid.any() and not np.asarray(eo["Tvalid"]).any()
    assert ((status & 32) != 0).all()
    zo, xs = [0.1, 0.3], [0.05, 0.4]
    G = api.closed_form_G(g, 1, 0.2, zo, xs, [0.0])
    Go = oracle.closed_form_G(o, 1, 0.2, zo, xs, [0.0])
    assert np.isfinite(G).all() and relerr(G, Go) < 1e-12
    assert np.array_equal(api.closed_form_G(g, 1, 0.2, zo, xs, [0.0], terms="scattered"), np.zeros_like(G))


@pytest.mark.parametrize("bad", [BiaxialMaterial(2.0 + 0.1j, 3.0, 0.0), BiaxialMaterial(2.0, complex(np.nan, 0), 3.0)],
                         ids=["eps33=0", "nan"])
def test_non_finite_general_layer_fails_the_build(oracle, bad):
    """A general-path (biaxial) layer with ε33 = 0 or a NaN entry: the reference's eigen
    raises for the first node and the build fails; the library returns the same message, and
    the oracle raises it too. A rule without nodes builds (no eigen call)."""
    import warnings
    from yellowthinfilms_b200 import api
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        st = [lay(IsotropicMaterial(1.0), 0.5), lay(bad, 0.3), lay(IsotropicMaterial(2.25), 0.5)]
    kr, wr = krho_grid(st[:1], W, kmax=3.0, width=1.0)
    ph, wp = uniform_phi(4)
    with pytest.raises(api.YTFError, match="matrix contains Infs or NaNs"):
        api.build_cavity_transfer_2d(st, W, 1, kr, wr, ph, wp, obs_layers=[1])
    with pytest.raises(RuntimeError, match="matrix contains Infs or NaNs"):
        oracle.build_cavity_transfer_2d(st, W, 1, kr, wr, ph, wp, obs_layers=[1], rotation=False)
    c = api.build_cavity_transfer_2d(st, W, 1, kr[:0], wr[:0], ph, wp, obs_layers=[1])
    assert c.n == 0


def test_bounded_pipeline_waits_run_out_and_the_context_survives(oracle):
    """With the poll limit at 1 every int8 tensor-core pipeline gives up at its first wait
    that is not already satisfied: closed_form_G raises instead of returning (2D lateral
    and 1D Bessel contractions). With the default limit back, the same context computes G,
    equal to the FP64 path to the int8x3 tolerance."""
    from yellowthinfilms_b200 import api
    from helpers import FOUNDATION_STACKS
    ctx = api.default_context()
    _, st = FOUNDATION_STACKS[3]
    kr, wr = krho_grid(st, W, kmax=10.0, width=0.5)
    ph, wp = uniform_phi(8)
    c2 = api.build_cavity_transfer_2d(st, W, 2, kr, wr, ph, wp, obs_layers=[2])
    xy = np.linspace(-0.3, 0.3, 12)
    _, st1 = FOUNDATION_STACKS[2]
    k1, w1 = krho_grid(st1, W, kmax=10.0, width=0.25)
    c1 = api.build_cavity_transfer_1d(st1, W, 2, k1, w1, obs_layers=[2])
    rho = np.geomspace(0.02, 2.0, 40)
    try:
        ctx.set_wait_limit(1)
        with pytest.raises(RuntimeError, match="timed out"):
            api.closed_form_G(c2, 2, 0.3, [0.1, 0.5], xy, xy, precision="int8x3")
        with pytest.raises(RuntimeError, match="timed out"):
            api.closed_form_G(c1, 2, 0.3, [0.1, 0.5], rho, [0.0], precision="int8x3")
    finally:
        ctx.set_wait_limit(0)
    G = api.closed_form_G(c2, 2, 0.3, [0.1, 0.5], xy, xy, precision="int8x3")
    assert relerr(G, api.closed_form_G(c2, 2, 0.3, [0.1, 0.5], xy, xy)) < 1e-6
    G1 = api.closed_form_G(c1, 2, 0.3, [0.1, 0.5], rho, [0.0], precision="int8x3")
    assert relerr(G1, api.closed_form_G(c1, 2, 0.3, [0.1, 0.5], rho, [0.0])) < 1e-6
