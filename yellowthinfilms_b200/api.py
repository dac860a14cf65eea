"""Python host API with the reference's names and argument meanings.

Mirrors the Julia entry points this library replaces:
  build_cavity_transfer_1d  (mod_CavityTransfer.jl:196-258)
  build_cavity_transfer_2d  (mod_CavityTransfer.jl:307-398)
  closed_form_G             (mod_ClosedFormField.jl:435-487, 711-753; lateral=:direct)
  gl_rule, halve_panels, build_kphi_grid, gausslegendre (mod_KxGrid.jl:361-394)
Layer indices are 1-based; G comes back as an (Nx, Ny, Nz, 3, 3) complex array indexed
G[x, y, z, field component, moment], exactly as the reference's Array{ComplexF64,5}.

Every call runs on the GPU through libytf.so; argument errors raise YTFError with the
reference's message text.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _native
from ._native import _i, _u8, addr, lib, ptr
from .materials import stack_arrays

TERMS = {"all": 0, "direct": 1, "scattered": 2, "toeplitz": 3, "hankel": 4}
PRECISION = {"fp64": 0, "split_bf16": 1, "int8x3": 2}


class YTFError(ValueError):
    """An argument error reported by libytf (the reference raises `error(...)` there)."""


class Context:
    """A libytf context: one CUDA device and the stream its calls run on."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        rc = lib().ytf_ctx_create(ctypes.byref(h), int(device))
        if rc != 0:
            raise RuntimeError(f"ytf_ctx_create(device={device}) failed with code {rc}: no usable CUDA device")
        self.h = h
        self.device = device

    def set_stream(self, cuda_stream: int) -> None:
        lib().ytf_ctx_set_stream(self.h, ctypes.c_void_p(int(cuda_stream)))

    def set_wait_limit(self, polls: int = 0) -> None:
        """Polls of each bounded wait in the int8 tensor-core pipelines before it gives up
        (0: the default); a wait that runs out makes the call raise RuntimeError."""
        self.check(lib().ytf_ctx_set_wait_limit(self.h, int(polls)))

    def set_group_bytes(self, nbytes: int = 0) -> None:
        """Workspace bound of one group of closed_form_G_batch's grouped 1D int8x3 synthesis
        (0: the default 4 GiB)."""
        self.check(lib().ytf_ctx_set_group_bytes(self.h, int(nbytes)))

    def sync(self) -> None:
        self.check(lib().ytf_ctx_sync(self.h))

    def error(self) -> str:
        return lib().ytf_last_error(self.h).decode()

    def profile(self, enable: bool = True) -> None:
        """Reset the per-kernel counters; time every launch with CUDA events if enabled."""
        self.check(lib().ytf_ctx_profile(self.h, int(bool(enable))))

    def profile_read(self) -> dict:
        """{kernel name: (summed event ms, launches)} since the last profile() call."""
        n = ctypes.c_int(0)
        self.check(lib().ytf_ctx_profile_read(self.h, 0, None, None, None, ctypes.byref(n)))
        m = max(n.value, 1)
        names = ctypes.create_string_buffer(32 * m)
        ms = np.zeros(m)
        launches = np.zeros(m, dtype=np.int64)
        self.check(lib().ytf_ctx_profile_read(self.h, m, names, ptr(ms), launches.ctypes.data_as(
            ctypes.POINTER(ctypes.c_long)), ctypes.byref(n)))
        raw = names.raw
        return {raw[32 * i:32 * i + 32].split(b"\0")[0].decode(): (float(ms[i]), int(launches[i])) for i in range(n.value)}

    def check(self, rc: int) -> None:
        if rc == 0:
            return
        msg = self.error()
        if rc == 1:
            raise YTFError(msg)
        raise RuntimeError(f"libytf error {rc}: {msg}")

    def __del__(self):
        if getattr(self, "h", None) is not None and getattr(_native, "_lib", None) is not None:
            _native._lib.ytf_ctx_destroy(self.h)
            self.h = None


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class Stack:
    """A stack uploaded to the device (layers of FlatOpticalLayer / FlatLayer)."""

    def __init__(self, layers, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.layers = list(layers)
        ek, mk, eps, mu, d = stack_arrays(self.layers)
        self._keep = (ek, mk, eps, mu, d)
        h = ctypes.c_void_p()
        rc = lib().ytf_stack_create(self.ctx.h, len(self.layers), ptr(ek, _i), ptr(mk, _i), ptr(eps.view(np.float64)),
                                    ptr(mu.view(np.float64)), ptr(d), ctypes.byref(h))
        self.ctx.check(rc)
        self.h = h

    def __len__(self):
        return len(self.layers)

    def __getitem__(self, i):
        return self.layers[i]

    def __del__(self):
        if getattr(self, "h", None) is not None and getattr(_native, "_lib", None) is not None:
            _native._lib.ytf_stack_destroy(self.h)
            self.h = None


def _as_stack(stack, ctx) -> Stack:
    if isinstance(stack, Stack):
        return stack
    return Stack(stack, ctx)


class _Cache:
    is2d = False

    def __init__(self, h, stack: Stack, omega, source_layer):
        self.h, self.stack, self.ctx = h, stack, stack.ctx
        self.omega, self.source_layer = float(omega), int(source_layer)
        n = ctypes.c_long()
        no = ctypes.c_int()
        obs = (ctypes.c_int * 32)()
        is2d = ctypes.c_int()
        rot = ctypes.c_int()
        lib().ytf_cache_info(h, ctypes.byref(n), ctypes.byref(no), obs, ctypes.byref(is2d), ctypes.byref(rot))
        self.n = int(n.value)
        self.obs_layers = [int(obs[i]) for i in range(no.value)]
        self.rotation = bool(rot.value)
        self.d_src = float(stack.layers[source_layer - 1].d)
        self.d_obs = {o: float(stack.layers[o - 1].d) for o in self.obs_layers}

    def __del__(self):
        # a cache lent by a BatchPlan (_plan set) belongs to the plan
        if (getattr(self, "h", None) is not None and getattr(_native, "_lib", None) is not None
                and getattr(self, "_plan", None) is None):
            _native._lib.ytf_cache_destroy(self.h)
        self.h = None

    def status(self):
        """(valid[n], Tvalid[n_obs, n], status bits[n]) as numpy arrays."""
        n, no = self.n, len(self.obs_layers)
        valid = np.zeros(n, np.uint8)
        tvalid = np.zeros(no * n, np.uint8)
        st = np.zeros(n, np.uint8)
        self.ctx.check(lib().ytf_cache_status(self.ctx.h, self.h, ptr(valid, _u8), ptr(tvalid, _u8), ptr(st, _u8)))
        return valid.astype(bool), tvalid.reshape(no, n).astype(bool), st

    @property
    def valid(self):
        return self.status()[0]

    @property
    def Tvalid(self):
        v = self.status()[1]
        return {o: v[i] for i, o in enumerate(self.obs_layers)}

    def export(self):
        """The cache's per-node arrays (T, Qf_src, Qb_src, sf, sb, basis) as numpy."""
        n, no = self.n, len(self.obs_layers)
        T = np.zeros(no * n * 32)
        Qf = np.zeros(4 * n)
        Qb = np.zeros(4 * n)
        sf = np.zeros(12 * n)
        sb = np.zeros(12 * n)
        basis = np.zeros(no * n * 32)
        self.ctx.check(lib().ytf_cache_export(self.ctx.h, self.h, ptr(T), ptr(Qf), ptr(Qb), ptr(sf), ptr(sb), ptr(basis)))
        c = lambda x: x.view(np.complex128)
        return dict(T=c(T).reshape(no, n, 4, 4).transpose(0, 1, 3, 2), Qf=c(Qf).reshape(n, 2), Qb=c(Qb).reshape(n, 2),
                    sf=c(sf).reshape(n, 3, 2).transpose(0, 2, 1), sb=c(sb).reshape(n, 3, 2).transpose(0, 2, 1),
                    basis=c(basis).reshape(no, n, 8, 2))


class CavityTransferCache1D(_Cache):
    """Device-resident CavityTransferCache1D (mod_CavityTransfer.jl:160-178)."""

    def __init__(self, h, stack, omega, source_layer, kx, wt):
        super().__init__(h, stack, omega, source_layer)
        self.kx_nodes, self.wt_nodes = kx, wt


class CavityTransferCache2D(_Cache):
    """Device-resident CavityTransferCache2D (mod_CavityTransfer.jl:273-294)."""
    is2d = True

    def __init__(self, h, stack, omega, source_layer, kr, wr, phi, wphi):
        super().__init__(h, stack, omega, source_layer)
        self.kr_nodes, self.kr_weights, self.phi_nodes, self.phi_weights = kr, wr, phi, wphi


def _f64(x):
    return np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.float64)))


def _obs_arg(obs_layers):
    if obs_layers is None:
        return 0, None
    a = np.ascontiguousarray(np.asarray(list(obs_layers), dtype=np.int32))
    return len(a), a


def build_cavity_transfer_1d(stack, omega, source_layer, kx_nodes, wt_nodes, obs_layers=None, check_symmetry=True,
                             ctx: Optional[Context] = None) -> CavityTransferCache1D:
    st = _as_stack(stack, ctx)
    kx, wt = _f64(kx_nodes), _f64(wt_nodes)
    if len(kx) != len(wt):
        raise YTFError("build_cavity_transfer_1d: kx_nodes/wt_nodes length mismatch")
    no, ob = _obs_arg(obs_layers)
    h = ctypes.c_void_p()
    rc = lib().ytf_transfer_1d(st.ctx.h, st.h, float(omega), int(source_layer), len(kx), ptr(kx), ptr(wt), no, ptr(ob, _i),
                               int(bool(check_symmetry)), ctypes.byref(h))
    st.ctx.check(rc)
    return CavityTransferCache1D(h, st, omega, source_layer, kx, wt)


def build_cavity_transfer_2d(stack, omega, source_layer, kr_nodes, kr_weights, phi_nodes, phi_weights, obs_layers=None,
                             rotation="auto", ctx: Optional[Context] = None) -> CavityTransferCache2D:
    st = _as_stack(stack, ctx)
    kr, wr, ph, wp = _f64(kr_nodes), _f64(kr_weights), _f64(phi_nodes), _f64(phi_weights)
    if len(kr) != len(wr):
        raise YTFError("build_cavity_transfer_2d: kρ nodes/weights length mismatch")
    if len(ph) != len(wp):
        raise YTFError("build_cavity_transfer_2d: φ nodes/weights length mismatch")
    rot = -1 if rotation == "auto" else int(bool(rotation))
    no, ob = _obs_arg(obs_layers)
    h = ctypes.c_void_p()
    rc = lib().ytf_transfer_2d(st.ctx.h, st.h, float(omega), int(source_layer), len(kr), ptr(kr), ptr(wr), len(ph), ptr(ph),
                               ptr(wp), no, ptr(ob, _i), rot, ctypes.byref(h))
    st.ctx.check(rc)
    return CavityTransferCache2D(h, st, omega, source_layer, kr, wr, ph, wp)


def closed_form_G(cache: _Cache, obs_layer: int, zsrc_local: float, z_obs, xs, ys, terms: str = "all",
                  precision: str = "fp64", out=None):
    """G[x, y, z, component, moment] of a point source (terms as the reference).

    ``precision`` selects the arithmetic of the 2D lateral sum: "fp64" (CUDA-core FP64),
    "split_bf16" (tensor cores, split-BF16 operands, FP32 accumulation) or "int8x3" (int8
    tensor cores, operands in three fixed-point base-256 digits, exact INT32 accumulation).
    For 1D caches "int8x3" also runs the Bessel contraction on the int8 tensor cores (on a
    deformed contour: the complex J_n's real and imaginary parts as two digit images);
    "split_bf16" keeps it FP64.

    ``out``: optional torch tensor (complex128, Nx*Ny*Nz*9 elements, Julia order) to write
    into instead of returning a new host array: a CUDA tensor (G stays on the device) or
    a pinned host tensor (G is copied back inside the call).
    """
    if terms not in TERMS:
        raise YTFError(f"closed_form_G: terms must be :all, :direct, :scattered, :toeplitz or :hankel (got :{terms})")
    zo, x, y = _f64(z_obs), _f64(xs), _f64(ys)
    nx, ny, nz = len(x), len(y), len(zo)
    ctx = cache.ctx
    if out is not None:
        if out.numel() != nx * ny * nz * 9:
            raise YTFError("closed_form_G: out has the wrong size")
        on_dev = int(bool(getattr(out, "is_cuda", False)))
        rc = lib().ytf_green(ctx.h, cache.h, int(obs_layer), float(zsrc_local), nz, ptr(zo), nx, ptr(x), ny, ptr(y),
                             TERMS[terms], PRECISION[precision], ctypes.c_void_p(out.data_ptr()), on_dev)
        ctx.check(rc)
        return out
    G = np.zeros(2 * 9 * nz * nx * ny)
    rc = lib().ytf_green(ctx.h, cache.h, int(obs_layer), float(zsrc_local), nz, ptr(zo), nx, ptr(x), ny, ptr(y),
                         TERMS[terms], PRECISION[precision], G.ctypes.data_as(ctypes.c_void_p), 0)
    ctx.check(rc)
    return G.view(np.complex128).reshape(3, 3, nz, ny, nx).transpose(4, 3, 2, 1, 0)


def cavity_response(stack, omega, s, kr, phi=0.0, ctx: Optional[Context] = None):
    """_cavity_response(stack, ω, s, kρ, φ) (mod_KSpaceFeatures.jl:109-127) at every kρ of
    ``kr`` (array), solved on the device."""
    st = _as_stack(stack, ctx)
    k = _f64(np.atleast_1d(kr))
    out = np.zeros(len(k))
    st.ctx.check(lib().ytf_cavity_response(st.ctx.h, st.h, float(omega), int(s), len(k), ptr(k), float(phi), ptr(out)))
    return out


def cavity_response_batch(items, phi=0.0, ctx: Optional[Context] = None):
    """cavity_response for many (stack, omega, source_layer, kr) tuples with one device
    synchronisation (ytf_cavity_response_batch). Returns one response array per item."""
    items = list(items)
    if not items:
        return []
    sts = [_as_stack(it[0], ctx) for it in items]
    ctx = ctx or sts[0].ctx
    ks = [_f64(np.atleast_1d(it[3])) for it in items]
    counts = np.array([len(k) for k in ks], np.int64)
    kall = _f64(np.concatenate(ks)) if counts.sum() else np.zeros(1)
    out = np.zeros(max(1, int(counts.sum())))
    hs = (ctypes.c_void_p * len(items))(*[st.h.value for st in sts])
    om = _f64([it[1] for it in items])
    src = np.array([int(it[2]) for it in items], np.int32)
    ctx.check(lib().ytf_cavity_response_batch(ctx.h, len(items), hs, ptr(om), ptr(src, _i),
                                              counts.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), ptr(kall),
                                              float(phi), ptr(out)))
    return np.split(out[:int(counts.sum())], np.cumsum(counts)[:-1])


def layer_light_lines(layer, omega, phi=0.0):
    """layer_light_lines(layer, ω, φ) (mod_KxGrid.jl:41-59): host arithmetic of libytf."""
    # ε and μ column-major, as stack_arrays lays out one layer
    eps = np.ascontiguousarray(np.asarray(layer.eps, np.complex128).T.reshape(9))
    mu = np.ascontiguousarray(np.asarray(layer.mu, np.complex128).T.reshape(9))
    out = np.zeros(3)
    n = ctypes.c_int(0)
    rc = lib().ytf_layer_light_lines(ptr(eps), ptr(mu), float(omega), float(phi), ptr(out), ctypes.byref(n))
    if rc != 0:
        raise YTFError("layer_light_lines: bad arguments")
    return out[:n.value].copy()


def point_kx_grid(stack, omega, source_layer, h_min, rho_max=0.0, target_decay=25.0, kr_cap=0.0, scan=True, order=8,
                  rtol=1e-6, ctx: Optional[Context] = None):
    """point_kx_grid (mod_ClosedFormGrid.jl:381-424) with the :fixed engine: (kx, wt, info).
    The pole scan's cavity responses are solved on the device; panels on the host; nodes by
    the device Gauss–Legendre expansion. ``poles``: (q, Γ) pairs to use instead of the scan
    (ytf_nodes_from_poles)."""
    return _grid(stack, omega, source_layer, h_min, rho_max, target_decay, kr_cap, scan, order, rtol, ctx, None)


def _grid(stack, omega, source_layer, h_min, rho_max, target_decay, kr_cap, scan, order, rtol, ctx, poles):
    from ._native import GridInfo, GridParams
    st = _as_stack(stack, ctx)
    prm = GridParams(float(h_min), float(rho_max), float(target_decay), float(kr_cap), int(bool(scan)), int(order),
                     float(rtol))
    info = GridInfo()
    n = ctypes.c_long(0)
    if poles is None:
        call = lambda cap, kp, wp: lib().ytf_nodes_1d(st.ctx.h, st.h, float(omega), int(source_layer), ctypes.byref(prm),
                                                      cap, kp, wp, ctypes.byref(n), ctypes.byref(info))
    else:
        pq = _f64([p[0] for p in poles]) if len(poles) else np.zeros(1)
        pg = _f64([p[1] for p in poles]) if len(poles) else np.zeros(1)
        call = lambda cap, kp, wp: lib().ytf_nodes_from_poles(st.ctx.h, st.h, float(omega), int(source_layer),
                                                              ctypes.byref(prm), len(poles), ptr(pq), ptr(pg), cap, kp,
                                                              wp, ctypes.byref(n), ctypes.byref(info))
    st.ctx.check(call(0, None, None))
    k = np.zeros(n.value)
    w = np.zeros(n.value)
    pan = np.zeros(2 * max(1, info.n_panels))
    info.panels = ptr(pan)
    info.panels_cap = info.n_panels
    st.ctx.check(call(n.value, ptr(k), ptr(w)))
    meta = dict(Kcut=info.Kcut, kmax=info.kmax, n_poles=info.n_poles, n_panels=info.n_panels,
                panels=pan[:2 * info.n_panels].reshape(-1, 2).copy(),
                poles=[(info.poles[i][0], info.poles[i][1]) for i in range(min(info.n_poles, 256))],
                light_lines=[info.light_lines[i] for i in range(min(info.n_light_lines, 64))])
    return k, w, meta


def adaptive_seeds(stack, omega, source_layer, h_min, rho_max=0.0, target_decay=25.0, kr_cap=0.0, scan=True,
                   rtol=1e-6, ctx: Optional[Context] = None):
    """adaptive_seeds(kspace_features(stack, ω, s; h_min, ρ_max, dims=1); rtol)
    (mod_KSpaceFeatures.jl:421-445): the adaptive engine's starting breakpoints."""
    from ._native import GridParams
    st = _as_stack(stack, ctx)
    prm = GridParams(float(h_min), float(rho_max), float(target_decay), float(kr_cap), int(bool(scan)), 8, float(rtol))
    n = ctypes.c_long(0)
    st.ctx.check(lib().ytf_adaptive_seeds(st.ctx.h, st.h, float(omega), int(source_layer), ctypes.byref(prm), 0, None,
                                          ctypes.byref(n)))
    out = np.zeros(n.value)
    st.ctx.check(lib().ytf_adaptive_seeds(st.ctx.h, st.h, float(omega), int(source_layer), ctypes.byref(prm), n.value,
                                          ptr(out), ctypes.byref(n)))
    return out


def point_krho_grid_2d(stack, omega, source_layer, h_min, rho_max, target_decay=25.0, kr_cap=0.0, scan=True, order=8,
                       rtol=1e-6, N_phi=None, N_phi_scan=32, ctx: Optional[Context] = None):
    """point_kρ_grid_2d (mod_ClosedFormGrid.jl:536-585) with the :fixed engine:
    (kρ, wρ, φ, wφ, info). kspace_features with dims = 2 scans the poles along every
    scanned direction on the device and sizes the uniform φ trapezoid (info["N_phi"]: the
    largest of 64, 2.5 Kcut ρ_max and the pole-track term, even); ``N_phi`` overrides it.
    One kρ rule serves every φ."""
    from ._native import GridInfo, GridParams
    st = _as_stack(stack, ctx)
    prm = GridParams(float(h_min), float(rho_max), float(target_decay), float(kr_cap), int(bool(scan)), int(order),
                     float(rtol))
    info = GridInfo()
    n, nphi = ctypes.c_long(0), ctypes.c_long(0)
    call = lambda cap, kp, wp: lib().ytf_nodes_2d(st.ctx.h, st.h, float(omega), int(source_layer), ctypes.byref(prm),
                                                  int(N_phi_scan), cap, kp, wp, ctypes.byref(n), ctypes.byref(nphi),
                                                  ctypes.byref(info))
    st.ctx.check(call(0, None, None))
    k = np.zeros(n.value)
    w = np.zeros(n.value)
    pan = np.zeros(2 * max(1, info.n_panels))
    info.panels = ptr(pan)
    info.panels_cap = info.n_panels
    st.ctx.check(call(n.value, ptr(k), ptr(w)))
    Np = int(nphi.value) if N_phi is None else int(N_phi)
    phi, wphi = build_kphi_grid(Np)
    meta = dict(Kcut=info.Kcut, kmax=info.kmax, n_poles=info.n_poles, n_panels=info.n_panels, N_phi=Np,
                N_phi_features=int(nphi.value), panels=pan[:2 * info.n_panels].reshape(-1, 2).copy(),
                poles=[(info.poles[i][0], info.poles[i][1]) for i in range(min(info.n_poles, 256))],
                light_lines=[info.light_lines[i] for i in range(min(info.n_light_lines, 64))])
    return k, w, phi, wphi, meta


def peaks_batch(ks, logR, prominence=np.log(1.05), floor_rel=1e-6):
    """Peaks (q, Γ) of many sampled log-responses at once (ytf_peaks_batch): ks and logR are
    [windows, points] arrays on log-uniform grids; returns one list of (q, Γ) per window."""
    K = np.ascontiguousarray(np.asarray(ks, np.float64))
    Y = np.ascontiguousarray(np.asarray(logR, np.float64))
    nw, npts = K.shape
    counts = np.zeros(max(nw, 1), np.int32)
    cap = nw * max(1, npts // 2)
    q, G = np.zeros(max(cap, 1)), np.zeros(max(cap, 1))
    tot = ctypes.c_long(0)
    rc = lib().ytf_peaks_batch(nw, npts, ptr(K), ptr(Y), float(prominence), float(floor_rel), cap, ptr(counts, _i),
                               ptr(q), ptr(G), ctypes.byref(tot))
    if rc != 0:
        raise YTFError("peaks_batch: bad arguments")
    cuts = np.cumsum(counts[:nw])[:-1]
    return [list(zip(a.tolist(), b.tolist())) for a, b in zip(np.split(q[:tot.value], cuts), np.split(G[:tot.value], cuts))]


def rule_panels(stack, omega, source_layer, h_min, rho_max=0.0, target_decay=25.0, kr_cap=0.0, scan=False, order=8,
                rtol=1e-6, poles=None, ctx: Optional[Context] = None):
    """The panels (an [n, 2] array) of point_kx_grid's rule (``poles`` given: of
    grid_from_poles's), host work only: the nodes of many rules then come from one
    gl_rule_batch call over (panels, singular) with the half-space light lines as singular
    points, bit for bit the nodes point_kx_grid / grid_from_poles return."""
    from ._native import GridInfo, GridParams
    st = _as_stack(stack, ctx)
    prm = GridParams(float(h_min), float(rho_max), float(target_decay), float(kr_cap), int(bool(scan)), int(order),
                     float(rtol))
    info = GridInfo()
    n = ctypes.c_long(0)
    if poles is None:
        call = lambda: lib().ytf_nodes_1d(st.ctx.h, st.h, float(omega), int(source_layer), ctypes.byref(prm), 0, None,
                                          None, ctypes.byref(n), ctypes.byref(info))
    else:
        pq = _f64([p[0] for p in poles]) if len(poles) else np.zeros(1)
        pg = _f64([p[1] for p in poles]) if len(poles) else np.zeros(1)
        call = lambda: lib().ytf_nodes_from_poles(st.ctx.h, st.h, float(omega), int(source_layer), ctypes.byref(prm),
                                                  len(poles), ptr(pq), ptr(pg), 0, None, None, ctypes.byref(n),
                                                  ctypes.byref(info))
    pan = np.zeros(2 * 16384)  # one call when the rule has at most 16384 panels (the panels are host work)
    info.panels = ptr(pan)
    info.panels_cap = 16384
    st.ctx.check(call())
    if info.n_panels > 16384:
        pan = np.zeros(2 * info.n_panels)
        info.panels = ptr(pan)
        info.panels_cap = info.n_panels
        st.ctx.check(call())
    return pan[:2 * info.n_panels].reshape(-1, 2).copy()


def bessel_j01(x, ctx: Optional[Context] = None):
    """(J_0(x), J_1(x)) of real x as the int8x3 1D synthesis evaluates them
    (ytf_bessel_j01: the CUDA library below |x| = 25, Hankel's asymptotic pair above)."""
    ctx = ctx or default_context()
    x = _f64(x)
    a, b = np.zeros(len(x)), np.zeros(len(x))
    ctx.check(lib().ytf_bessel_j01(ctx.h, len(x), ptr(x), ptr(a), ptr(b)))
    return a, b


def rule_panels_batch(problems, order=8, rtol=1e-6, target_decay=25.0, kr_cap=0.0, ctx: Optional[Context] = None):
    """rule_panels for many problems in one call (ytf_rule_panels_batch, host threads): each
    problem a dict with stack, omega, source_layer, h_min, rho_max and optionally poles
    ([(q, Γ)]: grid_from_poles's panels; absent or None: point_kx_grid's without the scan).
    Returns the [n, 2] panel arrays in order, each equal to its own rule_panels call."""
    from ._native import GridParams
    ctx = ctx or default_context()
    n = len(problems)
    if n == 0:
        return []
    sts = [_as_stack(P["stack"], ctx) for P in problems]
    hs = (ctypes.c_void_p * n)(*[st.h for st in sts])
    om = _f64([P["omega"] for P in problems])
    src = np.ascontiguousarray([int(P["source_layer"]) for P in problems], np.int32)
    prm = (GridParams * n)(*[GridParams(float(P["h_min"]), float(P.get("rho_max", 0.0)), float(target_decay),
                                        float(kr_cap), 0, int(order), float(rtol)) for P in problems])
    npl = np.ascontiguousarray([-1 if P.get("poles") is None else len(P["poles"]) for P in problems], np.int32)
    allp = [p for P in problems if P.get("poles") is not None for p in P["poles"]]
    q = _f64([p[0] for p in allp]) if allp else np.zeros(1)
    g = _f64([p[1] for p in allp]) if allp else np.zeros(1)
    counts = np.zeros(n, np.int64)
    total = ctypes.c_long(0)
    cap = max(16384, 4096 * n)
    for _ in range(2):
        buf = np.zeros(2 * cap)
        rc = lib().ytf_rule_panels_batch(ctx.h, n, hs, ptr(om), ptr(src, _i), prm, ptr(npl, _i), ptr(q), ptr(g), cap,
                                         ptr(buf), counts.ctypes.data_as(ctypes.POINTER(ctypes.c_long)),
                                         ctypes.byref(total))
        if rc == 0:
            break
        if total.value > cap:
            cap = int(total.value)
            continue
        ctx.check(rc)
    else:
        ctx.check(rc)
    cuts = np.cumsum(counts)[:-1]
    return [a.reshape(-1, 2) for a in np.split(buf[:2 * int(total.value)], 2 * cuts)]


class MLP:
    """The node-placement MLP on the device (ytf_mlp_*): widths sizes[0] -> ... -> 2, GELU
    between layers, BF16 weights with FP32 accumulation, trained by libytf's own forward,
    backward and Adam kernels."""

    def __init__(self, sizes=(154, 256, 256, 256, 256, 2), seed=0, device=0):
        self.sizes = [int(x) for x in sizes]
        arr = np.asarray(self.sizes, np.int32)
        h = ctypes.c_void_p()
        rc = lib().ytf_mlp_create(int(device), len(self.sizes) - 1, ptr(arr, _i), ctypes.c_ulonglong(seed),
                                  ctypes.byref(h))
        if rc != 0:
            raise YTFError(f"ytf_mlp_create failed ({rc})")
        self.h = h
        self.nparam = int(lib().ytf_mlp_num_params(h))

    def __del__(self):
        if getattr(self, "h", None) is not None and getattr(_native, "_lib", None) is not None:
            _native._lib.ytf_mlp_destroy(self.h)
            self.h = None

    def _check(self, rc):
        if rc != 0:
            raise YTFError(lib().ytf_mlp_last_error(self.h).decode())

    def set_stream(self, stream_handle):
        self._check(lib().ytf_mlp_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    @property
    def params(self):
        p = np.zeros(self.nparam, np.float32)
        self._check(lib().ytf_mlp_params(self.h, p.ctypes.data_as(ctypes.c_void_p), None))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparam
        self._check(lib().ytf_mlp_params(self.h, None, p.ctypes.data_as(ctypes.c_void_p)))

    def forward(self, X):
        """Outputs [B, 2] for inputs X [B, sizes[0]] (numpy, or a CUDA float32 tensor)."""
        if hasattr(X, "is_cuda") and X.is_cuda:
            import torch
            out = torch.empty((X.shape[0], 2), dtype=torch.float32, device=X.device)
            self._check(lib().ytf_mlp_forward(self.h, X.shape[0], ctypes.c_void_p(X.data_ptr()),
                                              ctypes.c_void_p(out.data_ptr()), 1))
            return out
        X = np.ascontiguousarray(X, np.float32)
        out = np.zeros((X.shape[0], 2), np.float32)
        self._check(lib().ytf_mlp_forward(self.h, X.shape[0], X.ctypes.data_as(ctypes.c_void_p),
                                          out.ctypes.data_as(ctypes.c_void_p), 0))
        return out

    def gradients(self, X, T):
        """(loss, gradient of the loss w.r.t. the parameter vector) for one batch (numpy)."""
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        g = np.zeros(self.nparam, np.float32)
        loss = ctypes.c_float(0)
        self._check(lib().ytf_mlp_gradients(self.h, X.shape[0], X.ctypes.data_as(ctypes.c_void_p),
                                            T.ctypes.data_as(ctypes.c_void_p), g.ctypes.data_as(ctypes.c_void_p),
                                            ctypes.byref(loss), 0))
        return float(loss.value), g

    def train(self, X, T, batch=4096, steps=100, lr=1e-3, seed=1, record=True):
        """Adam steps on mini-batches of the device-resident set X [n, d], T [n, 2] (CUDA float32
        tensors). Returns the per-step mini-batch losses (numpy) when ``record``."""
        losses = np.zeros(steps, np.float32) if record else None
        self._check(lib().ytf_mlp_train(self.h, X.shape[0], ctypes.c_void_p(X.data_ptr()),
                                        ctypes.c_void_p(T.data_ptr()), int(batch), int(steps), float(lr),
                                        ctypes.c_ulonglong(seed),
                                        losses.ctypes.data_as(ctypes.c_void_p) if record else None))
        return losses


def grid_from_poles(stack, omega, source_layer, poles, h_min, rho_max=0.0, target_decay=25.0, kr_cap=0.0, order=8,
                    rtol=1e-6, ctx: Optional[Context] = None):
    """The point rule with given real-axis poles (q, Γ) instead of the scan (ytf_nodes_from_poles)."""
    return _grid(stack, omega, source_layer, h_min, rho_max, target_decay, kr_cap, False, order, rtol, ctx, list(poles))


def contour_rule(k0, npanels=512, order=8, L=None, h=None, breaks=()):
    """Gauss–Legendre rule on the deformed path kρ(t) = t - i h sin(π t / L), t in [0, L]
    (defaults L = 20 k0, h = 0.05 k0: below the real axis, back on it at both ends). Returns
    complex nodes and weights (w = kρ'(t) w_t). ``breaks``: values of t in (0, L) where panels
    must end (the half-space light lines: the path passes closest to those branch points there,
    and a panel edge at them keeps the rule's convergence geometric); the npanels are shared
    among the segments in proportion to their lengths, uniform within each."""
    L = 20.0 * k0 if L is None else float(L)
    h = 0.05 * k0 if h is None else float(h)
    x, wx = gausslegendre(order)
    bs = sorted({0.0, L} | {float(b) for b in breaks if 0.0 < float(b) < L})
    if len(bs) == 2:
        edges = np.linspace(0.0, L, npanels + 1)
    else:
        seg = np.diff(bs)
        cnt = np.maximum(1, np.round(npanels * seg / L).astype(int))
        edges = np.unique(np.concatenate([np.linspace(a, b, n + 1) for a, b, n in zip(bs[:-1], bs[1:], cnt)]))
    c = 0.5 * (edges[1:] + edges[:-1])
    hw = 0.5 * np.diff(edges)
    t = (c[:, None] + hw[:, None] * x[None, :]).ravel()
    wt = (hw[:, None] * wx[None, :]).ravel()
    k = t - 1j * h * np.sin(np.pi * t / L)
    dk = 1.0 - 1j * h * (np.pi / L) * np.cos(np.pi * t / L)
    return k, dk * wt


def build_cavity_transfer_1d_contour(stack, omega, source_layer, k_nodes, w_nodes, obs_layers=None,
                                     ctx: Optional[Context] = None) -> CavityTransferCache1D:
    """build_cavity_transfer_1d on complex nodes of a deformed contour (ytf_transfer_1d_contour)."""
    st = _as_stack(stack, ctx)
    k = np.asarray(k_nodes, np.complex128)
    w = np.asarray(w_nodes, np.complex128)
    if len(k) != len(w):
        raise YTFError("build_cavity_transfer_1d: kx_nodes/wt_nodes length mismatch")
    kr, ki, wr, wi = (np.ascontiguousarray(a) for a in (k.real, k.imag, w.real, w.imag))
    no, ob = _obs_arg(obs_layers)
    h = ctypes.c_void_p()
    st.ctx.check(lib().ytf_transfer_1d_contour(st.ctx.h, st.h, float(omega), int(source_layer), len(k), ptr(kr),
                                               ptr(ki), ptr(wr), ptr(wi), no, ptr(ob, _i), ctypes.byref(h)))
    return CavityTransferCache1D(h, st, omega, source_layer, k, w)


def bessel_j(order, z, ctx: Optional[Context] = None):
    """J_order(z) for complex z on the device (the contour synthesis's Bessel functions)."""
    ctx = ctx or default_context()
    z = np.atleast_1d(np.asarray(z, np.complex128))
    zr, zi = np.ascontiguousarray(z.real), np.ascontiguousarray(z.imag)
    outr, outi = np.zeros(len(z)), np.zeros(len(z))
    ctx.check(lib().ytf_bessel_j(ctx.h, int(order), len(z), ptr(zr), ptr(zi), ptr(outr), ptr(outi)))
    return outr + 1j * outi


def build_cavity_transfer_batch(items, ctx: Optional[Context] = None):
    """Many caches in one call (ytf_transfer_batch): each item is a dict with the keyword
    arguments of build_cavity_transfer_1d (``kx_nodes``, ``wt_nodes``) or
    build_cavity_transfer_2d (``kr_nodes``, ``kr_weights``, ``phi_nodes``, ``phi_weights``),
    plus ``stack``, ``omega``, ``source_layer`` and optionally ``obs_layers``,
    ``check_symmetry`` (1D) and ``rotation`` (2D). The node solves of all items share the
    same kernel launches. Returns the caches in order."""
    from ._native import TransferDesc
    descs = (TransferDesc * max(1, len(items)))()
    keep, meta = [], []
    for i, it in enumerate(items):
        st = _as_stack(it["stack"], ctx)
        ctx = ctx or st.ctx
        is2d = "kr_nodes" in it
        if is2d:
            k, w = _f64(it["kr_nodes"]), _f64(it["kr_weights"])
            ph, wp = _f64(it["phi_nodes"]), _f64(it["phi_weights"])
            if len(ph) != len(wp):
                raise YTFError("build_cavity_transfer_2d: φ nodes/weights length mismatch")
        elif getattr(it["kx_nodes"], "is_cuda", False):
            # a device-resident rule (gl_rule_batch(device=True)): float64 CUDA tensors on
            # this context's GPU, read on its stream
            k, w = it["kx_nodes"], it["wt_nodes"]
            if k.dtype != w.dtype or str(k.dtype) != "torch.float64" or not (k.is_contiguous() and w.is_contiguous()):
                raise YTFError("build_cavity_transfer_1d: device nodes must be contiguous float64 CUDA tensors")
            ph = wp = np.zeros(0)
        else:
            k, w = _f64(it["kx_nodes"]), _f64(it["wt_nodes"])
            ph = wp = np.zeros(0)
        if len(k) != len(w):
            raise YTFError("build_cavity_transfer_%s: node/weight length mismatch" % ("2d" if is2d else "1d"))
        no, ob = _obs_arg(it.get("obs_layers"))
        rot = it.get("rotation", "auto")
        d = descs[i]
        d.stack = st.h
        d.omega = float(it["omega"])
        d.source_layer = int(it["source_layer"])
        d.nk = len(k)
        dev = hasattr(k, "data_ptr")
        d.k_nodes, d.k_weights = (k.data_ptr(), w.data_ptr()) if dev else (addr(k), addr(w))
        d.nodes_on_device = int(dev)
        d.nphi = len(ph)
        d.phi_nodes, d.phi_weights = addr(ph), addr(wp)
        d.nobs, d.obs_layers = no, addr(ob)
        d.check_symmetry = int(bool(it.get("check_symmetry", True)))
        d.rotation = -1 if rot == "auto" else int(bool(rot))
        d.is2d = int(is2d)
        keep += [k, w, ph, wp, ob]
        meta.append((st, is2d, k, w, ph, wp, it))
    hs = (ctypes.c_void_p * max(1, len(items)))()
    if items:
        ctx.check(lib().ytf_transfer_batch(ctx.h, len(items), descs, hs))
    out = []
    for i, (st, is2d, k, w, ph, wp, it) in enumerate(meta):
        h = ctypes.c_void_p(hs[i])
        if is2d:
            out.append(CavityTransferCache2D(h, st, it["omega"], it["source_layer"], k, w, ph, wp))
        else:
            out.append(CavityTransferCache1D(h, st, it["omega"], it["source_layer"], k, w))
    return out


def closed_form_G_batch(items, precision: str = "fp64"):
    """closed_form_G over many items with one synchronisation (ytf_green_batch). Each item is
    a tuple (cache, obs_layer, zsrc_local, z_obs, xs, ys) or a dict with those keys plus
    optional ``terms``, ``precision`` and ``out`` (as closed_form_G). Returns the G arrays
    (or the ``out`` tensors) in order."""
    from ._native import GreenDesc
    descs = (GreenDesc * max(1, len(items)))()
    keep, outs = [], []
    ctx = None
    for i, it in enumerate(items):
        if not isinstance(it, dict):
            it = dict(zip(("cache", "obs_layer", "zsrc_local", "z_obs", "xs", "ys"), it))
        cache = it["cache"]
        ctx = ctx or cache.ctx
        terms = it.get("terms", "all")
        if terms not in TERMS:
            raise YTFError(f"closed_form_G: terms must be :all, :direct, :scattered, :toeplitz or :hankel (got :{terms})")
        zo, x, y = _f64(it["z_obs"]), _f64(it["xs"]), _f64(it["ys"])
        nx, ny, nz = len(x), len(y), len(zo)
        out = it.get("out")
        if out is not None:
            if out.numel() != nx * ny * nz * 9:
                raise YTFError("closed_form_G: out has the wrong size")
            optr, on_dev = out.data_ptr(), int(bool(getattr(out, "is_cuda", False)))
            outs.append(out)
        else:
            G = np.zeros(2 * 9 * nz * nx * ny)
            optr, on_dev = G.ctypes.data, 0
            outs.append((G, nx, ny, nz))
        d = descs[i]
        d.cache, d.obs_layer, d.zsrc_local = cache.h, int(it["obs_layer"]), float(it["zsrc_local"])
        d.nz, d.z_obs, d.nx, d.xs, d.ny, d.ys = nz, addr(zo), nx, addr(x), ny, addr(y)
        d.terms, d.precision = TERMS[terms], PRECISION[it.get("precision", precision)]
        d.out, d.out_is_device = optr, on_dev
        keep += [zo, x, y]
    if items:
        ctx.check(lib().ytf_green_batch(ctx.h, len(items), descs))
    res = []
    for o in outs:
        if isinstance(o, tuple):
            G, nx, ny, nz = o
            res.append(G.view(np.complex128).reshape(3, 3, nz, ny, nx).transpose(4, 3, 2, 1, 0))
        else:
            res.append(o)
    return res


class BatchPlan:
    """An uneven batch prepared once and replayed as one CUDA graph (ytf_plan_*; no
    counterpart in the reference, whose callers loop build_cavity_transfer_* and
    closed_form_G per item). ``transfer_items`` as build_cavity_transfer_batch (``rotation``
    is ignored: 2D items take the full (kρ, φ) solve); ``green_items`` as closed_form_G_batch
    without ``cache`` (item i synthesises from the cache of transfer item i). Small
    observation sets share one batched FP64 synthesis kernel; larger 2D sets (or another
    precision) run closed_form_G's own kernels inside the same graph; 1D items are FP64.
    ``tune``: dict of ytf_tune fields (block, ctas_per_sm, tile, chunk, synth_ctas_per_sm)
    or None for the defaults. Every ``run`` re-reads the node, weight and coordinate arrays
    held by the plan (``inputs(i)`` returns them for in-place updates of the same sizes)."""

    def __init__(self, transfer_items, green_items, tune=None, ctx: Optional[Context] = None):
        from ._native import GreenDesc, TransferDesc
        if len(transfer_items) != len(green_items):
            raise YTFError("BatchPlan: transfer_items and green_items differ in length")
        nb = len(transfer_items)
        self._td = (TransferDesc * max(1, nb))()
        self._gd = (GreenDesc * max(1, nb))()
        self._keep, self._inputs, self._outs, self._meta = [], [], [], []
        for i, (it, g) in enumerate(zip(transfer_items, green_items)):
            st = _as_stack(it["stack"], ctx)
            ctx = ctx or st.ctx
            is2d = "kr_nodes" in it
            if is2d:
                k, w = _f64(it["kr_nodes"]), _f64(it["kr_weights"])
                ph, wp = _f64(it["phi_nodes"]), _f64(it["phi_weights"])
            else:
                k, w = _f64(it["kx_nodes"]), _f64(it["wt_nodes"])
                ph = wp = np.zeros(0)
            if len(k) != len(w) or len(ph) != len(wp):
                raise YTFError("BatchPlan: node/weight length mismatch (item %d)" % i)
            no, ob = _obs_arg(it.get("obs_layers"))
            d = self._td[i]
            d.stack, d.omega, d.source_layer = st.h, float(it["omega"]), int(it["source_layer"])
            d.nk, d.k_nodes, d.k_weights = len(k), addr(k), addr(w)
            d.nphi, d.phi_nodes, d.phi_weights = len(ph), addr(ph), addr(wp)
            d.nobs, d.obs_layers = no, addr(ob)
            d.check_symmetry = int(bool(it.get("check_symmetry", True)))
            d.rotation = 0
            d.is2d = int(is2d)
            if not isinstance(g, dict):
                g = dict(zip(("obs_layer", "zsrc_local", "z_obs", "xs", "ys"), g))
            terms = g.get("terms", "all")
            if terms not in TERMS:
                raise YTFError(f"closed_form_G: terms must be :all, :direct, :scattered, :toeplitz or :hankel (got :{terms})")
            prec = g.get("precision", "fp64")
            if prec not in PRECISION:
                raise YTFError(f"closed_form_G: unknown precision {prec!r}")
            zo, x, y = _f64(g["z_obs"]), _f64(g["xs"]), _f64(g["ys"])
            nx, ny, nz = len(x), len(y), len(zo)
            out = g.get("out")
            e = self._gd[i]
            if out is not None:
                if out.numel() != nx * ny * nz * 9:
                    raise YTFError("closed_form_G: out has the wrong size")
                e.out, e.out_is_device = out.data_ptr(), int(bool(getattr(out, "is_cuda", False)))
                self._outs.append(out)
            else:
                G = np.zeros(2 * 9 * max(nz * nx * ny, 1))
                e.out, e.out_is_device = G.ctypes.data, 0
                self._outs.append((G, nx, ny, nz))
            e.cache, e.obs_layer, e.zsrc_local = None, int(g["obs_layer"]), float(g["zsrc_local"])
            e.nz, e.z_obs, e.nx, e.xs, e.ny, e.ys = nz, addr(zo), nx, addr(x), ny, addr(y)
            e.terms, e.precision = TERMS[terms], PRECISION[prec]
            self._keep += [k, w, ph, wp, ob, zo, x, y]
            self._inputs.append(dict(k=k, w=w, phi=ph, wphi=wp, z=zo, x=x, y=y))
            self._meta.append((st, is2d, it))
        self.ctx = ctx or default_context()
        self.n_items = nb
        self.h = None
        h = ctypes.c_void_p()
        tp = self._tune_struct(tune)
        self.ctx.check(lib().ytf_plan_create(self.ctx.h, nb, self._td, self._gd, tp, ctypes.byref(h)))
        self.h = h
        self.tune = self._tune_dict(tune)

    @staticmethod
    def _tune_dict(tune):
        t = dict(block=128, ctas_per_sm=4, tile=1024, chunk=2048, synth_ctas_per_sm=2)
        t.update(tune or {})
        return t

    def _tune_struct(self, tune):
        from ._native import Tune
        if tune is None:
            return None
        t = self._tune_dict(tune)
        self._tune_c = Tune(t["block"], t["ctas_per_sm"], t["tile"], t["chunk"], t["synth_ctas_per_sm"])
        return ctypes.byref(self._tune_c)

    def retune(self, tune):
        """Re-record the graph with other tiles (caches, scratch and staging are kept)."""
        self.ctx.check(lib().ytf_plan_retune(self.h, self._tune_struct(tune or {})))
        self.tune = self._tune_dict(tune)

    def inputs(self, i: int) -> dict:
        """The arrays item i is read from at every run (k, w, phi, wphi, z, x, y)."""
        return self._inputs[i]

    def run(self):
        """Stage the inputs and launch the graph on the context's stream (asynchronous)."""
        self.ctx.check(lib().ytf_plan_run(self.h))

    def wait(self) -> float:
        """Synchronise, deliver the host outputs; returns the graph's device time in ms."""
        ms = ctypes.c_float()
        self.ctx.check(lib().ytf_plan_wait(self.h, ctypes.byref(ms)))
        return float(ms.value)

    def __call__(self):
        self.run()
        self.wait()
        return self.results()

    def results(self):
        """G of every item, as closed_form_G returns it (views of the plan's host buffers, or
        the ``out`` tensors)."""
        res = []
        for o in self._outs:
            if isinstance(o, tuple):
                G, nx, ny, nz = o
                res.append(G[:2 * 9 * nz * nx * ny].view(np.complex128).reshape(3, 3, nz, ny, nx).transpose(4, 3, 2, 1, 0))
            else:
                res.append(o)
        return res

    def cache(self, i: int):
        """The cache of item i (owned by the plan)."""
        h = ctypes.c_void_p()
        self.ctx.check(lib().ytf_plan_cache(self.h, int(i), ctypes.byref(h)))
        st, is2d, it = self._meta[i]
        inp = self._inputs[i]
        if is2d:
            c = CavityTransferCache2D(h, st, it["omega"], it["source_layer"], inp["k"], inp["w"], inp["phi"], inp["wphi"])
        else:
            c = CavityTransferCache1D(h, st, it["omega"], it["source_layer"], inp["k"], inp["w"])
        c._plan = self
        return c

    def info(self) -> dict:
        n, p, k, hi, ho = ctypes.c_long(), ctypes.c_int(), ctypes.c_int(), ctypes.c_long(), ctypes.c_long()
        self.ctx.check(lib().ytf_plan_info(self.h, ctypes.byref(n), ctypes.byref(p), ctypes.byref(k), ctypes.byref(hi),
                                           ctypes.byref(ho)))
        return dict(nodes=int(n.value), passes=int(p.value), kernels=int(k.value), h2d_bytes=int(hi.value),
                    d2h_bytes=int(ho.value))

    def close(self):
        if getattr(self, "h", None) is not None and getattr(_native, "_lib", None) is not None:
            _native._lib.ytf_plan_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()


def gausslegendre(n: int):
    x = np.zeros(n)
    w = np.zeros(n)
    if lib().ytf_gauss_legendre(int(n), ptr(x), ptr(w)) != 0:
        raise YTFError("gausslegendre: n must be ≥ 1")
    return x, w


def gl_rule(panels: Sequence, order: int = 8, singular=(), ctx: Optional[Context] = None):
    """Composite Gauss–Legendre rule on `panels` (mod_KxGrid.jl:361-384), on the device."""
    ctx = ctx or default_context()
    if isinstance(panels, np.ndarray):
        P = np.asarray(panels, np.float64).reshape(-1, 2)
        pa, pb = np.ascontiguousarray(P[:, 0]), np.ascontiguousarray(P[:, 1])
    else:
        pa = _f64([p[0] for p in panels]) if len(panels) else np.zeros(0)
        pb = _f64([p[1] for p in panels]) if len(panels) else np.zeros(0)
    s = _f64(list(singular)) if len(singular) else np.zeros(1)
    nodes = np.zeros(len(panels) * order)
    wts = np.zeros(len(panels) * order)
    ctx.check(lib().ytf_gl_rule(ctx.h, len(panels), ptr(pa), ptr(pb), int(order), len(singular), ptr(s), ptr(nodes),
                                ptr(wts)))
    return nodes, wts


def gl_rule_batch(sets, order: int = 8, ctx: Optional[Context] = None, device: bool = False):
    """gl_rule for many (panels, singular) sets with one device call (ytf_gl_rule_batch);
    panels as [n, 2] arrays or pair sequences. Returns [(nodes, weights)] in order, each equal
    to its own gl_rule call. With ``device`` the rules stay in device memory
    (ytf_gl_rule_batch_device): float64 CUDA tensors, views of one allocation, ready for
    build_cavity_transfer_batch on the context's stream."""
    ctx = ctx or default_context()
    if not sets:
        return []
    P = [np.asarray(p, np.float64).reshape(-1, 2) for p, _ in sets]
    S = [_f64(list(sg)) for _, sg in sets]
    npan = np.array([len(p) for p in P], np.int32)
    nsing = np.array([len(sg) for sg in S], np.int32)
    pa = _f64(np.concatenate([p[:, 0] for p in P])) if npan.sum() else np.zeros(1)
    pb = _f64(np.concatenate([p[:, 1] for p in P])) if npan.sum() else np.zeros(1)
    sg = _f64(np.concatenate(S)) if nsing.sum() else np.zeros(1)
    tot = int(npan.sum()) * order
    if device:
        import torch
        buf = torch.empty(2 * max(tot, 1), dtype=torch.float64, device=f"cuda:{ctx.device}")
        ctx.check(lib().ytf_gl_rule_batch_device(ctx.h, len(sets), ptr(npan, _i), ptr(pa), ptr(pb), int(order),
                                                 ptr(nsing, _i), ptr(sg), buf.data_ptr(), buf.data_ptr() + 8 * max(tot, 1)))
        sizes = (npan.astype(np.int64) * order).tolist()
        return list(zip(torch.split(buf[:tot], sizes), torch.split(buf[max(tot, 1):max(tot, 1) + tot], sizes)))
    nodes, wts = np.zeros(max(tot, 1)), np.zeros(max(tot, 1))
    ctx.check(lib().ytf_gl_rule_batch(ctx.h, len(sets), ptr(npan, _i), ptr(pa), ptr(pb), int(order), ptr(nsing, _i),
                                      ptr(sg), ptr(nodes), ptr(wts)))
    cuts = np.cumsum(npan.astype(np.int64) * order)[:-1]
    return list(zip(np.split(nodes[:tot], cuts), np.split(wts[:tot], cuts)))


def halve_panels(panels):
    """`panels` with every panel split in two (mod_KxGrid.jl:387-388). A [n, 2] array gives a
    [2n, 2] array (the same midpoints (a + b) / 2), a sequence of pairs a list of pairs."""
    if isinstance(panels, np.ndarray):
        P = np.asarray(panels, np.float64).reshape(-1, 2)
        m = (P[:, 0] + P[:, 1]) / 2
        out = np.empty((2 * len(P), 2))
        out[0::2, 0], out[0::2, 1] = P[:, 0], m
        out[1::2, 0], out[1::2, 1] = m, P[:, 1]
        return out
    out = []
    for a, b in panels:
        m = (a + b) / 2
        out += [(float(a), m), (m, float(b))]
    return out


def build_kphi_grid(N_phi: int):
    """Uniform trapezoid in φ (mod_KxGrid.jl:390-394)."""
    return np.array([2 * np.pi * p / N_phi for p in range(N_phi)]), np.full(N_phi, 2 * np.pi / N_phi)


def _noalloc_tensors(device: int, z_obs, xs, ys, out) -> None:
    """Refuse what ytf_green_noalloc would misread: it takes raw device addresses, so every
    tensor must be a contiguous CUDA tensor on the cache's device, the coordinates float64
    and ``out`` complex128."""
    import torch
    for name, t, dt in (("z_obs", z_obs, torch.float64), ("xs", xs, torch.float64), ("ys", ys, torch.float64),
                        ("out", out, torch.complex128)):
        if not isinstance(t, torch.Tensor):
            raise YTFError(f"closed_form_G_noalloc: {name} must be a torch tensor on cuda:{device}")
        if not t.is_cuda or t.device.index != device:
            raise YTFError(f"closed_form_G_noalloc: {name} must be on cuda:{device} (got {t.device})")
        if t.dtype != dt:
            raise YTFError(f"closed_form_G_noalloc: {name} must be {dt} (got {t.dtype})")
        if not t.is_contiguous():
            raise YTFError(f"closed_form_G_noalloc: {name} must be contiguous")


def closed_form_G_noalloc(cache: CavityTransferCache2D, obs_layer: int, zsrc_local: float, z_obs, xs, ys, out,
                          terms: str = "all"):
    """closed_form_G for a 2D cache that allocates no device memory inside the library.

    For hosts that keep all device memory in their own pool, or that must not trigger the
    device-wide synchronisation of cudaMalloc: the library's scratch is a fixed 64 MiB
    array (limit 9·nz·(n_nodes + Nx·Ny) ≤ 4,194,304 complex values). ``z_obs``, ``xs``,
    ``ys`` (float64) and ``out`` (complex128, Nx·Ny·Nz·9, Julia order) are contiguous CUDA
    tensors on the cache's device that the caller allocated; anything else raises
    YTFError. Concurrent calls on the GPU share the scratch and must be serialised by the
    caller; the first call on a device should precede any stream capture.
    """
    if terms not in TERMS:
        raise YTFError(f"closed_form_G: terms must be :all, :direct, :scattered, :toeplitz or :hankel (got :{terms})")
    _noalloc_tensors(cache.ctx.device, z_obs, xs, ys, out)
    nz, nx, ny = z_obs.numel(), xs.numel(), ys.numel()
    if out.numel() != nx * ny * nz * 9:
        raise YTFError("closed_form_G: out has the wrong size")
    v = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = lib().ytf_green_noalloc(cache.ctx.h, cache.h, int(obs_layer), float(zsrc_local), nz, v(z_obs), nx, v(xs), ny, v(ys),
                                 TERMS[terms], v(out))
    cache.ctx.check(rc)
    return out
