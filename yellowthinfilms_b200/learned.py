"""Learned node placement for the Sommerfeld k-quadrature (no counterpart in the reference).

The reference places its point-rule nodes from a scan of the source layer's cavity response
along the real kρ axis (kspace_features / real_axis_poles, mod_KSpaceFeatures.jl:151-360):
thousands of full stack solves, then golden-section and bisection refinements per peak. Here
a small MLP (libytf's ytf_mlp: 154 -> 256 x4 -> 2, GELU, BF16 weights, FP32 accumulation,
trained by libytf's own kernels) predicts that scanned curve — log R(k) and a pole-proximity
score — from a stack descriptor, the frequency and k. Its peaks are candidate poles; one
batched device call samples the EXACT response on a small window around every candidate,
which fixes each pole's (q, Γ) for fixed_kρ_rule (ytf_nodes_from_poles) in place of the
scan's thousands of samples and sequential refinement rounds. Every node of the resulting
rule is then solved exactly by the transfer path. A proposed rule (Gauss–Legendre order 8) is
accepted only if its G agrees to the requested tolerance with G on the same panels at order 10,
and the order-10 rule is returned; otherwise the rule of one exact scan of the response is
checked the same way, then refined by halving until two levels agree, the plain method's own
check (and the reference's scanned rule is the last resort).

Training data come from the solver itself: random stacks of the air / uniaxial film /
substrate form, each scanned on a log kρ grid by ytf_cavity_response on the device.
"""
from __future__ import annotations

import numpy as np

from . import api
from .materials import FlatOpticalLayer, IsotropicMaterial, UniaxialMaterial

MAX_LAYERS = 8
N_FEATURES = MAX_LAYERS * 19 + 2  # 154
LAMBDA_REF = 600.0                 # nm: frequency feature = λ_ref / λ
K_LO, K_HI = 0.25, 160.0           # scan range in units of k0 (covers Kcut = 25 / 20 nm at 450-750 nm)
LOG_SCALE = 4.0                    # target 0 = log R / LOG_SCALE


def film_stack(rng, lam=None):
    """A random stack of the air / uniaxial film / substrate form (nm): the film has
    εo = -U[1, 6] + i 10^U[-2.5, -0.3], εe = U[2, 6] + i 10^U[-2.7, -0.5] (losses from sharp to
    broad guided modes), d U[20, 100]; the substrate ε U[1.5, 4]; air is 200 nm above the
    film. Returns (stack, λ)."""
    if lam is None:
        lam = float(rng.uniform(450.0, 750.0))
    eo = complex(-rng.uniform(1.0, 6.0), 10 ** rng.uniform(-2.5, -0.3))
    ee = complex(rng.uniform(2.0, 6.0), 10 ** rng.uniform(-2.7, -0.5))
    st = [FlatOpticalLayer(IsotropicMaterial(1.0), 200.0),
          FlatOpticalLayer(UniaxialMaterial(eo, ee), float(rng.uniform(20.0, 100.0))),
          FlatOpticalLayer(IsotropicMaterial(float(rng.uniform(1.5, 4.0))), 100.0)]
    return st, lam


def scan_grid(k0, n):
    """n log-spaced kρ over [K_LO, K_HI] k0."""
    return k0 * np.exp(np.linspace(np.log(K_LO), np.log(K_HI), n))


def scan_grids(k0s, n):
    """scan_grid of every k0 (rows of an [len(k0s), n] array, the same products)."""
    return np.asarray(k0s, np.float64)[:, None] * np.exp(np.linspace(np.log(K_LO), np.log(K_HI), n))[None, :]


def feature_row(stack, k0):
    """The k-independent part of a feature row (float32 [154], last entry 0): per layer (up
    to 8) Re and Im of the 9 ε entries / 10 and the thickness in wavelengths; then λ_ref / λ."""
    row = np.zeros(N_FEATURES)
    for l, layer in enumerate(stack[:MAX_LAYERS]):
        e = np.asarray(layer.eps, np.complex128).T.reshape(9)  # column-major, as stack_arrays
        row[19 * l:19 * l + 9] = e.real / 10.0
        row[19 * l + 9:19 * l + 18] = e.imag / 10.0
        row[19 * l + 18] = float(layer.d) * k0 / (2 * np.pi)
    row[-2] = k0 * LAMBDA_REF / (2 * np.pi)
    return row.astype(np.float32)


def k_feature(k0, ks):
    """The last feature column, k / (K_HI k0) (float32)."""
    return (np.asarray(ks) / (K_HI * k0)).astype(np.float32)


def features(stack, k0, ks):
    """[len(ks), 154] float32: feature_row with k / (K_HI k0) as the last column."""
    X = np.empty((len(ks), N_FEATURES), np.float32)
    X[:] = feature_row(stack, k0)
    X[:, -1] = k_feature(k0, ks)
    return X


def peaks(ks, logR, prominence=np.log(1.05), floor_rel=1e-6):
    """Peaks of a sampled log-response (the scan's rule of real_axis_poles on samples): local
    maxima with prominence, position by a parabola through the three samples in log k, width
    Γ from the nearer half-power crossing (linear interpolation). Returns [(q, Γ)]."""
    y = np.asarray(logR, np.float64)
    n = len(y)
    if n < 3:
        return []
    ymin = max(y.max() + np.log(floor_rel), np.log(1e-10))
    lk = np.log(ks)
    step = lk[1] - lk[0]
    W = int(np.ceil(np.log(4.0) / step))
    out = []
    # local maxima above the floor (vectorised), then each candidate in order
    cand = np.nonzero((y[1:-1] > y[:-2]) & (y[1:-1] >= y[2:]) & (y[1:-1] >= ymin))[0] + 1
    for i in cand:
        i = int(i)
        lo, hi = max(0, i - W), min(n - 1, i + W)
        # the run of samples ≤ y[i] on each side (bounded by the ±W window)
        above = np.nonzero(y[lo:i] > y[i])[0]
        jl = lo + int(above[-1]) + 1 if len(above) else lo
        above = np.nonzero(y[i + 1:hi + 1] > y[i])[0]
        jr = i + int(above[0]) if len(above) else hi
        base = max(y[jl:i + 1].min(), y[i:jr + 1].min())
        if y[i] - base < prominence:
            continue
        den = y[i - 1] - 2 * y[i] + y[i + 1]
        off = 0.5 * (y[i - 1] - y[i + 1]) / den if den < 0 else 0.0
        q = float(np.exp(lk[i] + np.clip(off, -0.5, 0.5) * step))
        P = np.exp(y[i])
        lvl = np.log(np.exp(base) + (P - np.exp(base)) / np.sqrt(2.0))
        G = np.inf
        # the first sample at or below the half-power level on each side, interpolated
        # linearly in log k against its neighbour towards the peak
        for js, dj in ((np.arange(i - 1, jl - 1, -1), 1), (np.arange(i + 1, jr + 1), -1)):
            hit = np.nonzero(y[js] <= lvl)[0]
            if len(hit):
                j = int(js[hit[0]])
                prev = j + dj
                t = (y[prev] - lvl) / (y[prev] - y[j])
                kc = np.exp(lk[prev] + t * (lk[j] - lk[prev]))
                G = min(G, abs(kc - q))
        if np.isfinite(G) and G > 0:
            out.append((q, float(G)))
    return out


def pole_score(ks, poles):
    """Pole-proximity score: max over poles of exp(-((k - q) / (2Γ))²)."""
    s = np.zeros(len(ks))
    for q, G in poles:
        s = np.maximum(s, np.exp(-((np.asarray(ks) - q) / (2 * G)) ** 2))
    return s


def training_set(n_stacks, n_k=2048, seed=0, ctx=None):
    """(X [n_stacks n_k, 154], T [n_stacks n_k, 2]) from device scans of random film stacks
    (source in the air layer)."""
    rng = np.random.default_rng(seed)
    Xs, Ts = [], []
    for _ in range(n_stacks):
        st, lam = film_stack(rng)
        k0 = 2 * np.pi / lam
        ks = scan_grid(k0, n_k)
        R = api.cavity_response(st, k0, 1, ks, ctx=ctx)
        logR = np.log(np.maximum(R, 1e-12))
        Xs.append(features(st, k0, ks))
        Ts.append(np.stack([logR / LOG_SCALE, pole_score(ks, peaks(ks, logR))], 1).astype(np.float32))
    return np.concatenate(Xs), np.concatenate(Ts)


def new_network(seed=0, device=0):
    return api.MLP((N_FEATURES, 256, 256, 256, 256, 2), seed=seed, device=device)


def copy_network(net, device=0):
    """A network with net's parameters (its own buffers: one per concurrent share)."""
    c = new_network(device=device)
    c.params = net.params
    return c


def train(net, X, T, steps, batch=4096, lr=1e-3, seed=1):
    """Adam on the device-resident set; returns the mini-batch losses."""
    import torch
    Xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    Td = torch.from_numpy(np.ascontiguousarray(T)).cuda()
    losses = net.train(Xd, Td, batch=batch, steps=steps, lr=lr, seed=seed)
    torch.cuda.synchronize()
    return losses


def predict_batch(net, stacks, n_k=2048, chunk=256):
    """The network's outputs (float64 [len(stacks) n_k, 2]) on every (layers, k0) item's scan
    grid: the feature rows are repeated over the grid on the device (the same float32 inputs
    as features()), chunk items per forward."""
    import torch
    out = []
    for c0 in range(0, len(stacks), chunk):
        part = stacks[c0:c0 + chunk]
        rows = torch.from_numpy(np.stack([feature_row(st, k0) for st, k0 in part])).cuda()
        k0s = np.array([k0 for _, k0 in part], np.float64)
        # k_feature(k0, scan_grid(k0, n_k)) of every item, row by row the same operations
        kf = torch.from_numpy((scan_grids(k0s, n_k) / (K_HI * k0s)[:, None]).astype(np.float32)).cuda()
        X = rows[:, None, :].repeat(1, n_k, 1)
        X[:, :, -1] = kf
        out.append(net.forward(X.view(-1, N_FEATURES)).cpu().numpy().astype(np.float64))
    return np.concatenate(out) if out else np.zeros((0, 2))


def _score_candidates(ks, logit, cand, threshold=0.1):
    """cand plus the local maxima of the pole score σ(logit) above ``threshold`` that lie more
    than 2Γ from every candidate so far (in increasing k), each with Γ = 2e-3 k. A false
    candidate costs one exact window sampling; a missed pole costs a refinement level, so the
    threshold is low."""
    sc = 1.0 / (1.0 + np.exp(-np.asarray(logit, np.float64)))
    idx = np.nonzero((sc[1:-1] > threshold) & (sc[1:-1] >= sc[:-2]) & (sc[1:-1] > sc[2:]))[0] + 1
    cand = list(cand)
    for i in idx:
        if all(abs(ks[i] - q) > 2 * G for q, G in cand):
            cand.append((float(ks[i]), float(ks[i] * 2e-3)))
    return cand


def propose_poles(net, stack, k0, n_k=2048):
    """Candidate real-axis poles (q, Γ) from the network: peaks of its predicted response and
    maxima of its pole score (> 0.3) on a fine log grid."""
    ks = scan_grid(k0, n_k)
    out = net.forward(features(stack, k0, ks)).astype(np.float64)
    cand = api.peaks_batch(ks[None, :], out[None, :, 0] * LOG_SCALE, prominence=np.log(1.01))[0]
    return sorted(_score_candidates(ks, out[:, 1], cand))


def _windows(cand, n_local):
    """The log windows (±6 max(Γ/q, 3e-3), n_local points) around the candidates: wide enough
    for the network's position error, fine enough to resolve the pole's width. An array
    [len(cand), n_local]."""
    if not len(cand):
        return np.zeros((0, n_local))
    c = np.asarray(cand, np.float64).reshape(-1, 2)
    w = np.maximum(c[:, 1] / c[:, 0], 3e-3)
    t = np.linspace(-6.0, 6.0, n_local)
    return c[:, :1] * np.exp(w[:, None] * t[None, :])


def refine_poles(stack, k0, source_layer, cand, n_local=129, ctx=None):
    """(q, Γ) of each candidate from the EXACT cavity response sampled on a small log window
    around it (±6 max(Γ/q, 2e-3)), all windows in one device call; candidates whose window
    shows no peak are dropped."""
    if not cand:
        return []
    wins = _windows(cand, n_local)
    R = api.cavity_response(stack, k0, source_layer, wins.reshape(-1), ctx=ctx)
    return _poles_from_windows(wins, R, n_local)


def refine_poles_batch(items, n_local=129, ctx=None):
    """refine_poles for many (stack, k0, source_layer, cand) items: every window of every
    item in ONE device call (ytf_cavity_response_batch) and the peaks of all windows in one
    host call. Returns the poles per item."""
    wins = [_windows(c, n_local) for (_, _, _, c) in items]
    idx = [i for i, w in enumerate(wins) if len(w)]
    out = [[] for _ in items]
    if not idx:
        return out
    Rs = api.cavity_response_batch([(items[i][0], items[i][1], items[i][2], wins[i].reshape(-1)) for i in idx], ctx=ctx)
    K = np.concatenate([wins[i] for i in idx])
    Y = np.log(np.maximum(np.concatenate([np.asarray(R, np.float64).reshape(-1, n_local) for R in Rs]), 1e-12))
    pk = api.peaks_batch(K, Y)
    w0 = 0
    for i in idx:
        nw = len(wins[i])
        out[i] = _merge_peaks(pk[w0:w0 + nw])
        w0 += nw
    return out


def _merge_peaks(per_window):
    """The peaks of an item's windows, sorted and merged (windows of neighbouring candidates
    may find the same pole)."""
    found = sorted(p for pk in per_window for p in pk)
    merged = []
    for q, G in found:
        if merged and abs(q - merged[-1][0]) <= 1e-6 * q:
            continue
        merged.append((q, G))
    return merged


def _poles_from_windows(wins, R, n_local):
    """Every peak of the sampled response in each window (the peak rule of peaks(), run for
    all windows in one host call, api.peaks_batch), merged across windows."""
    if not len(wins):
        return []
    K = np.asarray(wins).reshape(-1, n_local)
    Y = np.log(np.maximum(np.asarray(R, np.float64)[:len(K) * n_local].reshape(len(K), n_local), 1e-12))
    return _merge_peaks(api.peaks_batch(K, Y))


def halved(stack, omega, panels, order, ctx=None):
    """The rule on the same panels split in two (the acceptance check), with the u²
    substitution at the half-space light lines as the original rule."""
    sing = sorted(set(api.layer_light_lines(stack[0], omega)) | set(api.layer_light_lines(stack[-1], omega)))
    p2 = api.halve_panels([tuple(p) for p in panels])
    return api.gl_rule(p2, order, singular=sing, ctx=ctx)


def learned_rule(net, stack, k0, source_layer, h_min, rho_max=0.0, order=8, rtol=1e-6, check=None, max_halvings=6,
                 ctx=None, check_order=10):
    """The learned point rule, with the plain method's refinement as the fallback.

    Proposes poles with the network, fixes them with one exact batched sampling, and builds
    fixed_kρ_rule on them. With ``check`` (a callable rule -> G) the rule is accepted when G
    agrees to rtol with G on the same panels at Gauss–Legendre order ``check_order`` (None:
    on the halved panels at ``order``); otherwise the proposal missed a pole and the
    plain method takes over: the rule of one exact scan of the response
    (exact_scan_poles_batch), checked the same way, then halved until two successive levels
    agree (max_halvings + 1 levels in all), and if they never do, the reference's scanned rule. On agreement the finer level
    of the agreeing pair is returned (its G is already computed and the more accurate of the
    two). Returns (k, w, info): info["learned"] is True when the proposed rule itself was
    accepted, info["halvings"] counts the levels past it, info["G"] is G on the returned rule
    when ``check`` was given."""
    poles = refine_poles(stack, k0, source_layer, propose_poles(net, stack, k0), ctx=ctx)
    k, w, info = api.grid_from_poles(stack, k0, source_layer, poles, h_min=h_min, rho_max=rho_max, order=order,
                                     rtol=rtol, ctx=ctx)
    info = dict(info, learned=True, halvings=0, proposed_poles=poles)
    if check is None:
        return k, w, info
    sing = sorted(set(api.layer_light_lines(stack[0], k0)) | set(api.layer_light_lines(stack[-1], k0)))
    panels = info["panels"]
    G = check(k, w)
    if check_order:
        panels2 = [tuple(p) for p in panels]
        kh, wh = api.gl_rule(panels2, check_order, singular=sing)
    else:
        panels2 = api.halve_panels([tuple(p) for p in panels])
        kh, wh = api.gl_rule(panels2, order, singular=sing)
    Gh = check(kh, wh)
    if np.linalg.norm(G - Gh) <= rtol * np.linalg.norm(Gh):
        info.update(learned=True, halvings=0, G=Gh, panels=np.asarray(panels2))
        return kh, wh, info
    # the proposal missed a pole: the rule of one exact scan, halved until two levels agree
    P = dict(stack=stack, layers=list(stack), k0=k0, source_layer=source_layer, h_min=h_min)
    poles = exact_scan_poles_batch([P], ctx=ctx)[0]
    k, w, info2 = api.grid_from_poles(stack, k0, source_layer, poles, h_min=h_min, rho_max=rho_max, order=order,
                                      rtol=rtol, ctx=ctx)
    panels = info2["panels"]
    G = check(k, w)
    for h in range(max_halvings + 1):
        if h == 0 and check_order:
            # the scanned rule's first check as the proposal's: the same panels at check_order
            panels2 = [tuple(p) for p in panels]
            kh, wh = api.gl_rule(panels2, check_order, singular=sing)
        else:
            panels2 = api.halve_panels([tuple(p) for p in panels])
            kh, wh = api.gl_rule(panels2, order, singular=sing)
        Gh = check(kh, wh)
        if np.linalg.norm(G - Gh) <= rtol * np.linalg.norm(Gh):
            # the check passed: return the finer of the two levels (already solved, and the
            # more accurate; its difference to the coarser one bounds the coarser one's error)
            info.update(learned=False, halvings=h + 1, G=Gh, panels=np.asarray(panels2))
            return kh, wh, info
        if not (h == 0 and check_order):
            panels, k, w, G = panels2, kh, wh, Gh
    k, w, info2 = api.point_kx_grid(stack, k0, source_layer, h_min=h_min, rho_max=rho_max, order=order, rtol=rtol,
                                    ctx=ctx)
    info.update(info2, learned=False, halvings=max_halvings + 2, G=check(k, w))
    return k, w, info


# ------------------------------------------------------------------------------------
# Batched forms: many problems (stack, k0, observation set) at once. Rules are built per
# problem; every G evaluation of a refinement level is ONE batched build and ONE batched
# synthesis over the problems still open (ytf_transfer_batch + ytf_green_batch), so the
# time follows the nodes solved rather than per-call latency.
# ------------------------------------------------------------------------------------
def batch_G(problems, rules, ctx=None, device=False):
    """G on each problem's rule: problems are dicts with stack (api.Stack or layers), k0,
    source_layer, zsrc_local, z (rows), rho (radii, on the x axis), terms and optionally the
    synthesis precision ("fp64" by default, "int8x3"); rules (k, w). With ``device`` the G
    arrays stay in device memory (complex128 CUDA tensors of the same (ρ, 1, z, 3, 3) shape)."""
    if not problems:
        return []
    caches = api.build_cavity_transfer_batch(
        [dict(stack=P["stack"], omega=P["k0"], source_layer=P["source_layer"], kx_nodes=k, wt_nodes=w,
              obs_layers=[P["source_layer"]]) for P, (k, w) in zip(problems, rules)], ctx=ctx)
    items = [dict(cache=c, obs_layer=P["source_layer"], zsrc_local=P["zsrc_local"], z_obs=P["z"], xs=P["rho"],
                  ys=[0.0], terms=P.get("terms", "all"), precision=P.get("precision", "fp64"))
             for P, c in zip(problems, caches)]
    if not device:
        return api.closed_form_G_batch(items)
    import torch
    shapes = [(len(P["rho"]), 1, len(P["z"])) for P in problems]
    outs = [torch.empty(nx * ny * nz * 9, dtype=torch.complex128, device="cuda") for nx, ny, nz in shapes]
    api.closed_form_G_batch([dict(it, out=o) for it, o in zip(items, outs)])
    return [o.view(3, 3, nz, ny, nx).permute(4, 3, 2, 1, 0) for o, (nx, ny, nz) in zip(outs, shapes)]


def _agree(pairs, rtol):
    """Per (G, G_halved) pair: ‖G - G_h‖ ≤ rtol ‖G_h‖ (numpy arrays, or device tensors with
    one host read for all pairs)."""
    if not pairs:
        return []
    if isinstance(pairs[0][1], np.ndarray):
        return [np.linalg.norm(a - b) <= rtol * np.linalg.norm(b) for a, b in pairs]
    import torch
    A = [a for a, _ in pairs]
    B = [b for _, b in pairs]
    # the norms of all pairs in a few multi-tensor launches (on the real views), one host read
    real = lambda xs: [torch.view_as_real(x) if x.is_complex() else x for x in xs]
    nd = torch.stack(torch._foreach_norm(real(torch._foreach_sub(A, B))))
    nb = torch.stack(torch._foreach_norm(real(B)))
    nrm = torch.stack([nd, nb], 1).cpu().numpy()
    return [bool(d <= rtol * n) for d, n in nrm]


def _sing(P):
    """The half-space light lines of problem P (the rule's u² points), kept in P["singular"]
    after the first call."""
    s = P.get("singular")
    if s is None:
        st = P["layers"]
        s = sorted(set(api.layer_light_lines(st[0], P["k0"])) | set(api.layer_light_lines(st[-1], P["k0"])))
        P["singular"] = s
    return s


def _refine_levels(problems, idx, rules, panels, G, rtol, max_halvings, order, ctx, out, device=False, solved=None,
                   check_order=None):
    """Halve the open problems' rules until G agrees with G on the halved rule (the plain
    method's own check), all open problems per batched level (the halved rules' nodes of a
    level in one ytf_gl_rule_batch call); fills out[i] = (G, k, w, halvings, converged) with
    the finer level of the agreeing pair (already solved, and the more accurate one). With G
    None the rules' own G and the first halved level are evaluated in one batch. ``solved``
    (optional list): solved[i] grows by the nodes of every rule problem i is solved and
    synthesised on. ``check_order`` (optional): the first level's finer rule is the same panels
    at that Gauss–Legendre order instead of the halved panels at ``order`` (fewer nodes for a
    higher degree of exactness); a problem that fails it keeps its order-``order`` rule and G,
    which the later levels halve. max_halvings + 1 levels in all."""
    open_ = list(idx)
    sing = {i: _sing(problems[i]) for i in open_}
    for h in range(max_halvings + 1):
        if not open_:
            break
        if h == 0 and check_order:
            p2s = [np.asarray(panels[i], np.float64).reshape(-1, 2) for i in open_]
            r2s = api.gl_rule_batch([(p2, sing[i]) for p2, i in zip(p2s, open_)], check_order, ctx=ctx, device=device)
        else:
            p2s = [api.halve_panels(np.asarray(panels[i], np.float64).reshape(-1, 2)) for i in open_]
            r2s = api.gl_rule_batch([(p2, sing[i]) for p2, i in zip(p2s, open_)], order, ctx=ctx, device=device)
        halv = {i: (p2, r2) for i, p2, r2 in zip(open_, p2s, r2s)}
        if solved is not None:
            for i in open_:
                solved[i] += len(halv[i][1][0]) + (len(rules[i][0]) if G is None else 0)
        if G is None:
            both = batch_G([problems[i] for i in open_] * 2, [rules[i] for i in open_] + [halv[i][1] for i in open_],
                           ctx=ctx, device=device)
            G = [None] * len(problems)
            for i, g in zip(open_, both[:len(open_)]):
                G[i] = g
            Gh = both[len(open_):]
        else:
            Gh = batch_G([problems[i] for i in open_], [halv[i][1] for i in open_], ctx=ctx, device=device)
        ok = _agree([(G[i], g) for i, g in zip(open_, Gh)], rtol)
        still = []
        for i, g, good in zip(open_, Gh, ok):
            if good:
                out[i] = (g, halv[i][1][0], halv[i][1][1], h, True)
                G[i] = None
            else:
                if not (h == 0 and check_order):
                    panels[i], rules[i], G[i] = halv[i][0], halv[i][1], g
                still.append(i)
        open_ = still
    for i in open_:
        out[i] = (G[i], rules[i][0], rules[i][1], max_halvings + 1, False)


def plain_rules_batch(problems, order=8, rtol=1e-6, max_halvings=8, ctx=None, device=False, solved=None):
    """The plain fixed rule (no pole knowledge: light-line breaks, u² substitution) of every
    problem, halved until two levels agree. Returns [(G, k, w, halvings, converged)]; with
    ``device`` every G (and the acceptance check) stays in device memory, and so do the
    rules (k, w as float64 CUDA tensors; a fallback rule of the scanned grid stays numpy);
    ``solved`` as _refine_levels."""
    panels = api.rule_panels_batch([dict(stack=P["stack"], omega=P["k0"], source_layer=P["source_layer"],
                                         h_min=P["h_min"], rho_max=P["rho_max"]) for P in problems], order=order, ctx=ctx)
    rules = api.gl_rule_batch([(p, _sing(P)) for p, P in zip(panels, problems)], order, ctx=ctx, device=device)
    out = [None] * len(problems)
    _refine_levels(problems, range(len(problems)), rules, panels, None, rtol, max_halvings, order, ctx, out, device,
                   solved)
    return out


def learned_rules_batch(net, problems, order=8, rtol=1e-6, max_halvings=6, ctx=None, device=False, build_rtol=None,
                        n_scan=2048, solved=None, pred=None, check_order=10):
    """learned_rule for every problem: the network over all problems' scan grids (features
    formed on the device), the exact window sampling of all problems in one device call,
    fixed_kρ_rule per problem, then the acceptance check; the rejected problems take the rule
    of one exact scan (exact_scan_poles_batch) refined in batched halving levels; a problem that
    never converges falls back to the reference's scanned rule. Returns [(G, k, w, accepted, halvings)]; ``device`` as plain_rules_batch.
    ``build_rtol`` (default rtol): the tolerance the proposed rules are built for; the
    acceptance check always uses rtol. ``n_scan``: points of the log grid the network is
    evaluated on per problem. ``solved`` as _refine_levels. ``pred``: the network's outputs on
    the problems' scan grids when already evaluated (predict_batch), else evaluated here.
    ``check_order``: the proposal's check compares its G with G on the same panels at this
    Gauss–Legendre order (10: 18 nodes solved per panel where the halving check takes 24, the
    order-10 rule returned on agreement; on panels sized for order 8 its error is a few
    percent of the order-8 rule's, which the agreement bounds), and so does the first level of
    a rejected problem's scanned rule; None checks by halving."""
    n_k = n_scan
    if pred is None:
        pred = predict_batch(net, [(P["layers"], P["k0"]) for P in problems], n_k)
    KS = scan_grids([P["k0"] for P in problems], n_k)
    pk = api.peaks_batch(KS, pred[:, 0].reshape(len(problems), n_k) * LOG_SCALE, prominence=np.log(1.01))
    cands = [sorted(_score_candidates(KS[j], pred[j * n_k:(j + 1) * n_k, 1], pk[j])) for j in range(len(problems))]
    polesets = refine_poles_batch([(P["stack"], P["k0"], P["source_layer"], c) for P, c in zip(problems, cands)], ctx=ctx)
    panels = api.rule_panels_batch([dict(stack=P["stack"], omega=P["k0"], source_layer=P["source_layer"],
                                         h_min=P["h_min"], rho_max=P["rho_max"], poles=poles)
                                    for P, poles in zip(problems, polesets)],
                                   order=order, rtol=rtol if build_rtol is None else build_rtol, ctx=ctx)
    rules = api.gl_rule_batch([(p, _sing(P)) for p, P in zip(panels, problems)], order, ctx=ctx, device=device)
    out = [None] * len(problems)
    # the proposals' own check (one level); a rejected proposal missed a pole: its rule comes
    # from one exact log scan of the response instead (batched over the rejected problems),
    # checked the same way, then refined by halving until two levels agree
    _refine_levels(problems, range(len(problems)), rules, panels, None, rtol, 0, order, ctx, out, device, solved,
                   check_order=check_order)
    rej = [i for i, r in enumerate(out) if not r[4]]
    if rej:
        scanned = exact_scan_poles_batch([problems[i] for i in rej], ctx=ctx)
        for i, pn in zip(rej, api.rule_panels_batch(
                [dict(stack=problems[i]["stack"], omega=problems[i]["k0"], source_layer=problems[i]["source_layer"],
                      h_min=problems[i]["h_min"], rho_max=problems[i]["rho_max"], poles=poles)
                 for i, poles in zip(rej, scanned)], order=order, rtol=rtol, ctx=ctx)):
            panels[i] = pn
        for i, r in zip(rej, api.gl_rule_batch([(panels[i], _sing(problems[i])) for i in rej], order, ctx=ctx,
                                               device=device)):
            rules[i] = r
        sub = [None] * len(problems)
        _refine_levels(problems, rej, rules, panels, None, rtol, max_halvings, order, ctx, sub, device, solved,
                       check_order=check_order)
        for i in rej:
            g, k, w, h, conv = sub[i]
            out[i] = (g, k, w, h + 1, conv)
    fall = [i for i, r in enumerate(out) if not r[4]]
    if fall:
        fr = []
        for i in fall:
            P = problems[i]
            k, w, _ = api.point_kx_grid(P["stack"], P["k0"], P["source_layer"], h_min=P["h_min"],
                                        rho_max=P["rho_max"], order=order, rtol=rtol, ctx=ctx)
            fr.append((k, w))
        if solved is not None:
            for i, (k, _) in zip(fall, fr):
                solved[i] += len(k)
        Gf = batch_G([problems[i] for i in fall], fr, ctx=ctx, device=device)
        for i, (k, w), g in zip(fall, fr, Gf):
            out[i] = (g, k, w, out[i][3], False)
    return [(g, k, w, conv and h == 0, h) for (g, k, w, h, conv) in out]


def concurrent_shares(fn, shares, ctxs, streams):
    """fn(share, ctx) for every share at once, one host thread per share, each with its own
    libytf context and CUDA stream (the thread's current torch stream too): while one share
    waits on the GPU (the library calls release the interpreter lock), another does its host
    work, so the host steps of a method (peaks, panels, levels) overlap the device work of the
    other shares. The problems of a share must use its context's Stack objects, and fn must not
    share other stateful objects between threads (an MLP's forward: evaluate the network before,
    learned_rules_batch(pred=...), or give each share its own copy_network). Returns the
    results in share order; the first exception of any share is raised after all finish."""
    import threading
    import torch
    out, err = [None] * len(shares), [None] * len(shares)

    def work(j):
        try:
            with torch.cuda.stream(streams[j]):
                out[j] = fn(shares[j], ctxs[j])
        except BaseException as e:  # re-raised in the calling thread
            err[j] = e
    ths = [threading.Thread(target=work, args=(j,)) for j in range(len(shares))]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for e in err:
        if e is not None:
            raise e
    return out


def exact_scan_poles_batch(problems, step=1e-3, n_local=129, ctx=None):
    """Real-axis poles (q, Γ) of every problem from its exact cavity response: one log scan from
    half the lowest light line to Kcut = min(max(target 25 / h_min, 2 kmax), 1e5 kmax) at
    relative step ``step`` (the reference's scan grid, mod_KSpaceFeatures.jl:151-204), the
    peaks of the sampled curve (prominence 1.05, light lines excluded), then exact windows
    around them for the widths the scan step cannot resolve: two batched device calls in all,
    in place of the reference's sequential refinement rounds."""
    items, grids = [], []
    for P in problems:
        st = P["layers"]
        ll = sorted({float(x) for L in st for x in api.layer_light_lines(L, P["k0"])})
        kmax = ll[-1] if ll else P["k0"]
        kcut = min(max(25.0 / P["h_min"], 2.0 * kmax), 1e5 * kmax)
        k_lo = 0.5 * (ll[0] if ll else P["k0"])
        n = int(np.floor(np.log(kcut / k_lo) / step + 1e-10)) + 1
        ks = k_lo * np.exp(step * np.arange(n))
        grids.append((ks, ll))
        items.append((P["stack"], P["k0"], P["source_layer"], ks))
    Rs = api.cavity_response_batch(items, ctx=ctx)
    cands = []
    for (ks, ll), R in zip(grids, Rs):
        pk = api.peaks_batch(ks[None, :], np.log(np.maximum(R, 1e-300))[None, :])[0]
        cands.append([(q, G) for q, G in pk if all(abs(q - L) > 1e-6 * q for L in ll)])
    return refine_poles_batch([(P["stack"], P["k0"], P["source_layer"], c) for P, c in zip(problems, cands)],
                              n_local=n_local, ctx=ctx)


def uniform_rule(k0, kmax, npanels, order=8):
    """The plain fixed grid: npanels equal Gauss-Legendre panels on [0, kmax]."""
    edges = np.linspace(0.0, kmax, npanels + 1)
    return api.gl_rule(list(zip(edges[:-1], edges[1:])), order)
