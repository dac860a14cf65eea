"""Guided-mode / plasmon pole-residue extraction on the deformed contour (no counterpart in the
reference, whose kρ path is the real axis: mod_ClosedFormGrid.jl:72-77).

The reference places narrow panels around each real-axis pole A/(kρ - q - iΓ) it scans
(mod_KSpaceFeatures.jl:142-145, 151-204). On the deformed contour kρ(t) = t - i h sin(π t / L)
a pole of a lossy stack sits above the path, at distance Γ + h sin(π q / L); when that is small
next to the panel width, the quadrature of the pole's part converges slowly. Singularity
subtraction removes it: near a simple pole k_p the integrand g(kρ) of G (for every (ρ, z) entry)
is Res_p / (kρ - k_p) + a function analytic at k_p, and

    ∫_C g dk = Σ_k w_k g(k_k) + Σ_p Res_p [ (Log(L - k_p) - Log(-k_p)) - Σ_k w_k / (k_k - k_p) ]

where the bracket is the exact integral of 1/(kρ - k_p) along the contour minus the rule's
value of it (the contour runs below the pole, so k - k_p stays in the lower half plane and the
principal logarithm is continuous along it). What is left for the rule is the analytic
remainder, which needs far fewer nodes.

Everything is evaluated by the CUDA path in FP64 on complex nodes (ytf_transfer_1d_contour +
closed_form_G): the pole k_p is refined from a real-axis estimate q + iΓ by the moment ratio
k_p = ∮ k g dk / ∮ g dk on a small circle (exact for one simple pole plus an analytic part; the
circle's trapezoid rule converges geometrically), and Res_p(ρ, z) = (1/2πi) ∮ g dk is one
closed_form_G call on the circle's nodes with weights (k_j - k_p)/m. On complex nodes the two
half-spaces take the proper sheet (the decaying wave), so g there is the analytic continuation
of its real-axis values on both sides of the axis. Circles must enclose one pole and no branch
point: radius below the distance to the half-space light lines and to the next pole.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import api


def circle_rule(center: complex, radius: float, m: int = 32, moment: int = 0):
    """Nodes k_j = c + r e^{iθ_j}, θ_j = 2π (j + ½)/m, and weights w_j = (k_j - c) k_j^moment / m:
    Σ_j w_j f(k_j) is the trapezoid rule of (1/2πi) ∮ f(k) k^moment dk."""
    th = 2 * np.pi * (np.arange(m) + 0.5) / m
    u = radius * np.exp(1j * th)
    k = center + u
    return k, u * k ** moment / m


def _circle_G(stack, omega, source_layer, obs_layer, zsrc, z_obs, xs, ys, k, w, terms, ctx):
    c = api.build_cavity_transfer_1d_contour(stack, omega, source_layer, k, w, obs_layers=[obs_layer], ctx=ctx)
    return api.closed_form_G(c, obs_layer, zsrc, z_obs, xs, ys, terms=terms)


def refine_pole(stack, omega: float, source_layer: int, guess: complex, radius: float, probe: dict, m: int = 32,
                max_iter: int = 30, tol: float = 1e-13, ctx: Optional[api.Context] = None) -> Tuple[complex, float]:
    """The complex pole inside the circle of ``radius`` around ``guess``, by the moment ratio
    ∮ k g dk / ∮ g dk at the probe entry with the largest residue (probe: dict with obs_layer,
    zsrc, z_obs, xs, ys of a small observation set). The circle follows the estimate until it
    moves by less than tol |k_p|. Raises ValueError when the circle holds no pole (the residue
    vanishes) or the estimate leaves the circle. Returns (k_p, radius)."""
    c = complex(guess)
    args = (probe["obs_layer"], probe["zsrc"], probe["z_obs"], probe["xs"], probe["ys"])
    for _ in range(max_iter):
        k, w0 = circle_rule(c, radius, m, 0)
        _, w1 = circle_rule(c, radius, m, 1)
        R = _circle_G(stack, omega, source_layer, *args, k, w0, "scattered", ctx)
        M1 = _circle_G(stack, omega, source_layer, *args, k, w1, "scattered", ctx)
        i = np.unravel_index(np.argmax(np.abs(R)), R.shape)
        if not (np.isfinite(R[i]) and np.isfinite(M1[i]) and np.abs(R[i]) > 0):
            raise ValueError(f"refine_pole: no pole inside the circle |k - {c:.6g}| = {radius:.3g}")
        kn = complex(M1[i] / R[i])
        if abs(kn - c) > radius:
            raise ValueError(f"refine_pole: the estimate {kn:.6g} left the circle around {c:.6g}")
        done = abs(kn - c) <= tol * abs(kn)
        c = kn
        if done:
            return c, radius
    return c, radius


def contour_poles(stack, omega: float, source_layer: int, estimates: Sequence[Tuple[float, float]], probe: dict,
                  branch_points: Sequence[float] = (), m: int = 32, ctx: Optional[api.Context] = None
                  ) -> List[Tuple[complex, float]]:
    """Complex poles from real-axis estimates (q, Γ) (the pole scan of point_kx_grid, or the
    learned proposals): each circle starts at q + iΓ/2 with a radius of at most Γ and half the
    distance to the neighbouring estimates, and must lie wholly right of the largest branch
    point (the half-space light lines): left of it the real axis is a half-space's propagating
    region, where the decaying-wave sheet has its cut (Im Q = 0) and a leaky pole lives on the
    other sheet, so such estimates are left to the rule. Estimates whose circle holds no pole
    are dropped. Returns [(k_p, r)] with r the circle used for the residue."""
    est = sorted((float(q), float(G)) for q, G in estimates)
    L_max = max(branch_points) if len(branch_points) else 0.0
    out = []
    for i, (q, G) in enumerate(est):
        r = G
        for j in (i - 1, i + 1):
            if 0 <= j < len(est):
                r = min(r, 0.5 * abs(est[j][0] - q))
        ctr = complex(q, 0.5 * G)
        r = min(r, 0.9 * (q - L_max))
        if not r > 0:
            continue
        try:
            kp, rr = refine_pole(stack, omega, source_layer, ctr, r, probe, m=m, ctx=ctx)
        except ValueError:
            continue
        if kp.imag > 0 and kp.real - rr > L_max and all(abs(kp - o[0]) > 1e-8 * abs(kp) for o in out):
            out.append((kp, rr))
    return out


def residues(stack, omega: float, source_layer: int, poles: Sequence[Tuple[complex, float]], obs_layer: int,
             zsrc_local: float, z_obs, xs, ys, terms: str = "all", m: int = 32, ctx: Optional[api.Context] = None):
    """Res_p G(x, y, z) (array of closed_form_G's shape) of every pole: (1/2πi) ∮ g dk on its
    circle, one closed_form_G call each."""
    out = []
    for kp, r in poles:
        k, w = circle_rule(kp, r, m, 0)
        out.append(_circle_G(stack, omega, source_layer, obs_layer, zsrc_local, z_obs, xs, ys, k, w, terms, ctx))
    return out


def pole_corrections(k_nodes, w_nodes, poles: Sequence[Tuple[complex, float]], k_start: complex = 0.0,
                     k_end: Optional[complex] = None) -> np.ndarray:
    """(Log(k_end - k_p) - Log(k_start - k_p)) - Σ_k w_k / (k_k - k_p) per pole: the exact
    integral of 1/(k - k_p) along the contour minus the rule's value of it."""
    k = np.asarray(k_nodes, np.complex128)
    w = np.asarray(w_nodes, np.complex128)
    ke = complex(k_end) if k_end is not None else complex(k[-1].real + 0.0, 0.0)
    out = []
    for kp, _ in poles:
        exact = np.log(ke - kp) - np.log(complex(k_start) - kp)
        out.append(exact - np.sum(w / (k - kp)))
    return np.asarray(out)


def closed_form_G_contour(cache, obs_layer: int, zsrc_local: float, z_obs, xs, ys, poles=(), terms: str = "all",
                          k_end: Optional[float] = None, m: int = 32):
    """closed_form_G on a deformed-contour cache with the given poles extracted: the rule's G
    plus Res_p (exact - rule) of each pole's 1/(k - k_p) part. The contour runs from 0 to
    ``k_end`` on the real axis (default 20 k0, contour_rule's)."""
    G = api.closed_form_G(cache, obs_layer, zsrc_local, z_obs, xs, ys, terms=terms)
    if not len(poles):
        return G
    kend = complex(k_end) if k_end is not None else complex(20.0 * cache.omega)
    corr = pole_corrections(cache.kx_nodes, cache.wt_nodes, poles, 0.0, kend)
    R = residues(cache.stack, cache.omega, cache.source_layer, poles, obs_layer, zsrc_local, z_obs, xs, ys, terms=terms,
                 m=m, ctx=cache.ctx)
    for c, r in zip(corr, R):
        G = G + c * r
    return G
