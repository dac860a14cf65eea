"""ctypes front end of the CPU FP64 oracle (``oracle/ytf_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA path. Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this module; the
product (``yellowthinfilms_b200``) never does.

Stacks are passed duck-typed: a sequence of layers, each with ``eps_kind``, ``mu_kind``
(0 isotropic, 1 uniaxial, 2 biaxial, 3 general 3x3), ``eps`` and ``mu`` (3x3 complex
arrays) and ``d``. Layer indices are 1-based, as in the reference's Julia API.

The general (biaxial / gyrotropic) mode solve calls LAPACK's own ZGEEVX, taken from
scipy's bundled LAPACK, with the arguments Julia's ``LinearAlgebra.eigen`` uses
(``geevx!('B','N','V','N')``), then sorts by (real, imag) as ``eigsortby`` does.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import build as _build  # noqa: E402

_lib = None

TERMS = {"all": 0, "direct": 1, "scattered": 2, "toeplitz": 3, "hankel": 4}

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)
_u8 = ctypes.POINTER(ctypes.c_ubyte)


def _zgeevx_pointer() -> int:
    import scipy.linalg.cython_lapack as cl
    cap = cl.__pyx_capi__["zgeevx"]
    get_name = ctypes.pythonapi.PyCapsule_GetName
    get_name.restype = ctypes.c_char_p
    get_name.argtypes = [ctypes.py_object]
    get_ptr = ctypes.pythonapi.PyCapsule_GetPointer
    get_ptr.restype = ctypes.c_void_p
    get_ptr.argtypes = [ctypes.py_object, ctypes.c_char_p]
    return get_ptr(cap, get_name(cap))


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = ctypes.CDLL(path)
        L.ytfo_last_error.restype = ctypes.c_char_p
        L.ytfo_set_zgeevx.argtypes = [ctypes.c_void_p]
        L.ytfo_cache_build.restype = ctypes.c_void_p
        L.ytfo_cache_build.argtypes = [ctypes.c_int, _i, _i, _d, _d, _d, ctypes.c_double, ctypes.c_int, ctypes.c_int, _i,
                                       ctypes.c_int, ctypes.c_int, _d, _d, ctypes.c_int, _d, _d, ctypes.c_int]
        L.ytfo_cache_free.argtypes = [ctypes.c_void_p]
        L.ytfo_cache_export.argtypes = [ctypes.c_void_p, _u8, _u8, _d, _d, _d, _d, _d, _d]
        L.ytfo_green.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _d, ctypes.c_int, _d,
                                 ctypes.c_int, _d, ctypes.c_int, _d]
        L.ytfo_amplitude_at.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _d, _d]
        L.ytfo_cavity_response.restype = ctypes.c_double
        L.ytfo_own_reflectance.restype = ctypes.c_double
        L.ytfo_own_reflectance.argtypes = [ctypes.c_int, _i, _i, _d, _d, _d, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.ytfo_cavity_response.argtypes = [ctypes.c_int, _i, _i, _d, _d, _d, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double]
        L.ytfo_set_zgeevx(ctypes.c_void_p(_zgeevx_pointer()))
        _lib = L
    return _lib


def _p(a, t=_d):
    return a.ctypes.data_as(t)


def _err():
    return lib().ytfo_last_error().decode()


def set_threads(n: int) -> None:
    lib().ytfo_set_threads(int(n))


def num_threads() -> int:
    return int(lib().ytfo_num_threads())


class _StackArrays:
    """Flat arrays of a duck-typed stack (kinds, column-major 3x3 tensors, thicknesses)."""

    def __init__(self, stack):
        nL = len(stack)
        self.nL = nL
        self.ek = np.array([int(l.eps_kind) for l in stack], dtype=np.int32)
        self.mk = np.array([int(l.mu_kind) for l in stack], dtype=np.int32)
        self.eps = np.ascontiguousarray(
            np.stack([np.asarray(l.eps, dtype=np.complex128).T.reshape(9) for l in stack]).view(np.float64))
        self.mu = np.ascontiguousarray(
            np.stack([np.asarray(l.mu, dtype=np.complex128).T.reshape(9) for l in stack]).view(np.float64))
        self.d = np.array([float(l.d) for l in stack], dtype=np.float64)

    def args(self):
        return (ctypes.c_int(self.nL), _p(self.ek, _i), _p(self.mk, _i), _p(self.eps), _p(self.mu), _p(self.d))


def _c(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def berreman(layer, w, kx, ky):
    a = _StackArrays([layer])
    out = np.zeros(32)
    lib().ytfo_berreman(ctypes.c_int(a.ek[0]), ctypes.c_int(a.mk[0]), _p(a.eps), _p(a.mu), ctypes.c_double(w),
                        ctypes.c_double(kx), ctypes.c_double(ky), _p(out))
    return out.view(np.complex128).reshape(4, 4, order="F")


def modes_stack(stack, w, kx, ky=0.0):
    a = _StackArrays(stack)
    out = np.zeros(72 * a.nL)
    rc = lib().ytfo_modes_stack(*a.args(), ctypes.c_double(w), ctypes.c_double(kx), ctypes.c_double(ky), _p(out))
    if rc != 0:
        raise RuntimeError(_err())
    z = out.view(np.complex128).reshape(a.nL, 36)
    res = []
    for l in range(a.nL):
        r = z[l]
        res.append(dict(Vf=r[0:8].reshape(4, 2, order="F"), Vb=r[8:16].reshape(4, 2, order="F"),
                        Wf=r[16:24].reshape(4, 2, order="F"), Wb=r[24:32].reshape(4, 2, order="F"),
                        Qf=r[32:34].copy(), Qb=r[34:36].copy()))
    return res


def s_all(stack, w, kx, ky=0.0):
    a = _StackArrays(stack)
    sl = np.zeros(32 * a.nL); sr = np.zeros(32 * a.nL); si = np.zeros(32 * max(a.nL - 1, 1))
    rc = lib().ytfo_s_all(*a.args(), ctypes.c_double(w), ctypes.c_double(kx), ctypes.c_double(ky), _p(sl), _p(sr), _p(si))
    if rc != 0:
        raise RuntimeError(_err())
    f = lambda x, n: x.view(np.complex128)[: 16 * n].reshape(n, 4, 4).transpose(0, 2, 1)
    return f(sl, a.nL), f(sr, a.nL), f(si, a.nL - 1)


def foundation(stack, w, kx, ky, layer, q, z):
    """T^o·[S₊;S₋] and its direct reference (Modal_amp / Modal_amp_profile) per obs layer."""
    a = _StackArrays(stack)
    tu = np.zeros(8 * a.nL); ref = np.zeros(8 * a.nL); sn = np.zeros(1)
    rc = lib().ytfo_foundation(*a.args(), ctypes.c_double(w), ctypes.c_double(kx), ctypes.c_double(ky), ctypes.c_int(layer),
                               ctypes.c_int(q), ctypes.c_double(z), _p(tu), _p(ref), _p(sn))
    if rc != 0:
        raise RuntimeError(_err())
    return tu.view(np.complex128).reshape(a.nL, 4), ref.view(np.complex128).reshape(a.nL, 4), float(sn[0])


class OracleCache:
    """Handle of a CavityTransferCache1D/2D built by the oracle."""

    def __init__(self, h, stack, w, src, obs, is2d, nk, np_, kr, wr, phi=None, wphi=None):
        self.h, self.stack, self.omega, self.source_layer = h, stack, w, src
        self.obs_layers, self.is2d, self.Nk, self.Np = obs, is2d, nk, np_
        self.kr, self.wr, self.phi, self.wphi = kr, wr, phi, wphi

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ytfo_cache_free(ctypes.c_void_p(self.h))
            self.h = None

    @property
    def n(self):
        return self.Nk * self.Np

    def export(self):
        n, no = self.n, len(self.obs_layers)
        valid = np.zeros(n, np.uint8); tvalid = np.zeros(no * n, np.uint8)
        T = np.zeros(no * n * 32); Qf = np.zeros(4 * n); Qb = np.zeros(4 * n)
        sf = np.zeros(12 * n); sb = np.zeros(12 * n); basis = np.zeros(no * n * 32)
        lib().ytfo_cache_export(ctypes.c_void_p(self.h), _p(valid, _u8), _p(tvalid, _u8), _p(T), _p(Qf), _p(Qb), _p(sf),
                                _p(sb), _p(basis))
        c = lambda x: x.view(np.complex128)
        return dict(valid=valid.astype(bool), Tvalid=tvalid.reshape(no, n).astype(bool),
                    T=c(T).reshape(no, n, 4, 4).transpose(0, 1, 3, 2), Qf=c(Qf).reshape(n, 2), Qb=c(Qb).reshape(n, 2),
                    sf=c(sf).reshape(n, 3, 2).transpose(0, 2, 1), sb=c(sb).reshape(n, 3, 2).transpose(0, 2, 1),
                    basis=c(basis).reshape(no, n, 8, 2))


def _obs(stack, obs_layers):
    N = len(stack)
    obs = sorted(set(range(1, N + 1) if obs_layers is None else [int(o) for o in obs_layers]))
    if not all(1 <= o <= N for o in obs):
        raise ValueError(f"obs_layers out of range 1:{N}")
    return obs


def build_cavity_transfer_1d(stack, omega, source_layer, kx_nodes, wt_nodes, obs_layers=None):
    a = _StackArrays(stack)
    obs = _obs(stack, obs_layers)
    kx, wt = _c(kx_nodes), _c(wt_nodes)
    ob = np.array(obs, dtype=np.int32)
    h = lib().ytfo_cache_build(*a.args(), ctypes.c_double(omega), ctypes.c_int(source_layer), ctypes.c_int(len(obs)),
                               _p(ob, _i), 0, ctypes.c_int(len(kx)), _p(kx), _p(wt), 0, None, None, -1)
    if not h:
        raise RuntimeError(_err())
    return OracleCache(h, stack, omega, source_layer, obs, False, len(kx), 1, kx, wt)


def build_cavity_transfer_2d(stack, omega, source_layer, kr_nodes, kr_weights, phi_nodes, phi_weights, obs_layers=None,
                             rotation="auto"):
    a = _StackArrays(stack)
    obs = _obs(stack, obs_layers)
    kr, wr, ph, wp = _c(kr_nodes), _c(kr_weights), _c(phi_nodes), _c(phi_weights)
    ob = np.array(obs, dtype=np.int32)
    rot = -1 if rotation == "auto" else int(bool(rotation))
    h = lib().ytfo_cache_build(*a.args(), ctypes.c_double(omega), ctypes.c_int(source_layer), ctypes.c_int(len(obs)),
                               _p(ob, _i), 1, ctypes.c_int(len(kr)), _p(kr), _p(wr), ctypes.c_int(len(ph)), _p(ph), _p(wp),
                               rot)
    if not h:
        raise RuntimeError(_err())
    return OracleCache(h, stack, omega, source_layer, obs, True, len(kr), len(ph), kr, wr, ph, wp)


def closed_form_G(cache, obs_layer, zsrc_local, z_obs, xs, ys, terms="all"):
    """G as an (Nx, Ny, Nz, 3, 3) array (field component, moment), Julia's layout."""
    zo, x, y = _c(np.atleast_1d(z_obs)), _c(np.atleast_1d(xs)), _c(np.atleast_1d(ys))
    G = np.zeros(2 * 9 * len(zo) * len(x) * len(y))
    rc = lib().ytfo_green(ctypes.c_void_p(cache.h), ctypes.c_int(obs_layer), ctypes.c_double(zsrc_local),
                          ctypes.c_int(len(zo)), _p(zo), ctypes.c_int(len(x)), _p(x), ctypes.c_int(len(y)), _p(y),
                          ctypes.c_int(TERMS[terms]), _p(G))
    if rc != 0:
        raise RuntimeError(_err())
    return G.view(np.complex128).reshape(3, 3, len(zo), len(y), len(x)).transpose(4, 3, 2, 1, 0)


def amplitude_at(cache, obs_layer, zsrc_local, seeds="all"):
    n = cache.n
    Af = np.zeros(12 * n); Ab = np.zeros(12 * n)
    s = {"all": 0, "f": 1, "b": 2}[seeds]
    rc = lib().ytfo_amplitude_at(ctypes.c_void_p(cache.h), ctypes.c_int(obs_layer), ctypes.c_double(zsrc_local),
                                 ctypes.c_int(s), _p(Af), _p(Ab))
    if rc != 0:
        raise RuntimeError(_err())
    return Af.view(np.complex128).reshape(n, 2, 3), Ab.view(np.complex128).reshape(n, 2, 3)


def gauss_legendre(n):
    x = np.zeros(n); w = np.zeros(n)
    lib().ytfo_gauss_legendre(ctypes.c_int(n), _p(x), _p(w))
    return x, w


def gl_rule(panels, order=8, singular=()):
    pa = _c([p[0] for p in panels]); pb = _c([p[1] for p in panels]); s = _c(list(singular) or [np.nan])
    nodes = np.zeros(len(panels) * order); wts = np.zeros(len(panels) * order)
    lib().ytfo_gl_rule(ctypes.c_int(len(panels)), _p(pa), _p(pb), ctypes.c_int(order), ctypes.c_int(len(singular)), _p(s),
                       _p(nodes), _p(wts))
    return nodes, wts


def light_lines(layer, omega, phi):
    a = _StackArrays([layer])
    out = np.zeros(8); n = ctypes.c_int(0)
    lib().ytfo_light_lines(ctypes.c_int(a.ek[0]), ctypes.c_int(a.mk[0]), _p(a.eps), _p(a.mu), ctypes.c_double(omega),
                           ctypes.c_double(phi), _p(out), ctypes.byref(n))
    return out[: n.value].copy()


def material_class(layer):
    a = _StackArrays([layer])
    c = lib().ytfo_material_class(ctypes.c_int(a.ek[0]), ctypes.c_int(a.mk[0]), _p(a.eps), _p(a.mu))
    return ["dielectric", "metallic", "hyperbolic", "gyrotropic"][c]


def cavity_response(stack, omega, s, kr, phi=0.0):
    a = _StackArrays(stack)
    return float(lib().ytfo_cavity_response(*a.args(), ctypes.c_double(omega), ctypes.c_int(s), ctypes.c_double(kr),
                                            ctypes.c_double(phi)))


def fixed_grid_1d(stack, omega, source_layer, h_min, rho_max=0.0, target_decay=25.0, kr_cap=0.0, scan=True, order=8,
                  rtol=1e-6):
    """kspace_features(dims=1) + fixed_kρ_rule: (nodes, weights, info)."""
    a = _StackArrays(stack)
    n = ctypes.c_int(0); info = np.zeros(4)
    args = (*a.args(), ctypes.c_double(omega), ctypes.c_int(source_layer), ctypes.c_double(h_min), ctypes.c_double(rho_max),
            ctypes.c_double(target_decay), ctypes.c_double(kr_cap), ctypes.c_int(int(scan)), ctypes.c_int(order),
            ctypes.c_double(rtol))
    rc = lib().ytfo_fixed_grid_1d(*args, None, None, ctypes.byref(n), _p(info))
    if rc != 0:
        raise RuntimeError(_err())
    nodes = np.zeros(n.value); wts = np.zeros(n.value)
    lib().ytfo_fixed_grid_1d(*args, _p(nodes), _p(wts), ctypes.byref(n), _p(info))
    return nodes, wts, dict(Kcut=info[0], kmax=info[1], n_poles=int(info[2]), n_panels=int(info[3]))


def adaptive_seeds(stack, omega, source_layer, h_min, rho_max=0.0, target_decay=25.0, kr_cap=0.0, scan=True, rtol=1e-6):
    """adaptive_seeds(kspace_features(dims=1); rtol)."""
    a = _StackArrays(stack)
    n = ctypes.c_int(0)
    args = (*a.args(), ctypes.c_double(omega), ctypes.c_int(source_layer), ctypes.c_double(h_min), ctypes.c_double(rho_max),
            ctypes.c_double(target_decay), ctypes.c_double(kr_cap), ctypes.c_int(int(scan)), ctypes.c_double(rtol))
    if lib().ytfo_adaptive_seeds(*args, None, ctypes.byref(n)) != 0:
        raise RuntimeError(_err())
    out = np.zeros(n.value)
    lib().ytfo_adaptive_seeds(*args, _p(out), ctypes.byref(n))
    return out


def fixed_grid_2d(stack, omega, source_layer, h_min, rho_max=0.0, target_decay=25.0, kr_cap=0.0, scan=True, order=8,
                  rtol=1e-6, n_phi_scan=32):
    """point_kρ_grid_2d: kspace_features(dims=2) + fixed_kρ_rule: (kρ nodes, weights, info)
    with info["N_phi"] the φ trapezoid's size."""
    a = _StackArrays(stack)
    n = ctypes.c_int(0); info = np.zeros(5)
    args = (*a.args(), ctypes.c_double(omega), ctypes.c_int(source_layer), ctypes.c_double(h_min), ctypes.c_double(rho_max),
            ctypes.c_double(target_decay), ctypes.c_double(kr_cap), ctypes.c_int(int(scan)), ctypes.c_int(order),
            ctypes.c_double(rtol), ctypes.c_int(n_phi_scan))
    rc = lib().ytfo_fixed_grid_2d(*args, None, None, ctypes.byref(n), _p(info))
    if rc != 0:
        raise RuntimeError(_err())
    nodes = np.zeros(n.value); wts = np.zeros(n.value)
    lib().ytfo_fixed_grid_2d(*args, _p(nodes), _p(wts), ctypes.byref(n), _p(info))
    return nodes, wts, dict(Kcut=info[0], kmax=info[1], n_poles=int(info[2]), n_panels=int(info[3]), N_phi=int(info[4]))


def own_reflectance(stack, k0, theta_deg, pol):
    a = _StackArrays(stack)
    return float(lib().ytfo_own_reflectance(*a.args(), ctypes.c_double(k0), ctypes.c_double(theta_deg),
                                            ctypes.c_int(1 if pol == "s" else 0)))


def strengths_2d(cache, obs_layer, zsrc_local, z, terms="all"):
    """Per-node strengths S[n, c + 3q] of one z-row and the node (kx, ky) of a 2D cache."""
    n = cache.n
    S = np.zeros(18 * n); kx = np.zeros(n); ky = np.zeros(n)
    rc = lib().ytfo_strengths_2d(ctypes.c_void_p(cache.h), ctypes.c_int(obs_layer), ctypes.c_double(zsrc_local),
                                 ctypes.c_double(z), ctypes.c_int(TERMS[terms]), _p(S), _p(kx), _p(ky))
    if rc != 0:
        raise RuntimeError(_err())
    return S.view(np.complex128).reshape(n, 9), kx, ky
