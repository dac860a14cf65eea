"""Host logic of the learned node placement (no GPU): the peak finder on sampled
log-responses (the scan's rule of real_axis_poles, mod_KSpaceFeatures.jl:151-204, on
samples) against a sample-by-sample restatement of the same walk."""
import numpy as np


def _peaks_loop(ks, logR, prominence=np.log(1.05), floor_rel=1e-6):
    y = np.asarray(logR, np.float64)
    n = len(y)
    if n < 3:
        return []
    ymin = max(y.max() + np.log(floor_rel), np.log(1e-10))
    lk = np.log(ks)
    step = lk[1] - lk[0]
    W = int(np.ceil(np.log(4.0) / step))
    out = []
    for i in range(1, n - 1):
        if not (y[i] > y[i - 1] and y[i] >= y[i + 1] and y[i] >= ymin):
            continue
        lo, hi = max(0, i - W), min(n - 1, i + W)
        jl = i
        while jl > lo and y[jl - 1] <= y[i]:
            jl -= 1
        jr = i
        while jr < hi and y[jr + 1] <= y[i]:
            jr += 1
        base = max(y[jl:i + 1].min(), y[i:jr + 1].min())
        if y[i] - base < prominence:
            continue
        den = y[i - 1] - 2 * y[i] + y[i + 1]
        off = 0.5 * (y[i - 1] - y[i + 1]) / den if den < 0 else 0.0
        q = float(np.exp(lk[i] + np.clip(off, -0.5, 0.5) * step))
        P = np.exp(y[i])
        lvl = np.log(np.exp(base) + (P - np.exp(base)) / np.sqrt(2.0))
        G = np.inf
        for rng_ in (range(i, jl - 1, -1), range(i, jr + 1)):
            prev = None
            for j in rng_:
                if y[j] <= lvl and prev is not None:
                    t = (y[prev] - lvl) / (y[prev] - y[j])
                    kc = np.exp(lk[prev] + t * (lk[j] - lk[prev]))
                    G = min(G, abs(kc - q))
                    break
                prev = j
        if np.isfinite(G) and G > 0:
            out.append((q, float(G)))
    return out


def test_peaks_equal_the_sample_walk():
    """learned.peaks (vectorised walks) returns exactly the (q, Γ) list of the sample-by-sample
    walk: Lorentzian peaks of several widths on a sloped background, with noise, plateaus, a
    peak next to the last sample, fine and coarse grids."""
    from yellowthinfilms_b200 import learned as L
    rng = np.random.default_rng(12)
    cases = found = 0
    for n in (129, 700, 2048, 4096):
        for trial in range(12):
            ks = np.exp(np.linspace(np.log(0.25), np.log(20.0), n))
            y = -0.3 * np.log(ks)
            for _ in range(int(rng.integers(0, 5))):
                q, g, a = rng.uniform(0.3, 19.0), 10 ** rng.uniform(-3, -0.5), rng.uniform(0.5, 40.0)
                y = y + np.log1p(a / (1 + ((ks - q) / g) ** 2))
            if trial % 3 == 1:
                y = y + rng.normal(0.0, 0.02, n)
            if trial % 3 == 2:
                y = np.round(y, 1)  # plateaus: equal neighbours
            if trial == 5:
                y[-2] = y.max() + 1.0
            got = L.peaks(ks, y)
            assert got == _peaks_loop(ks, y), (n, trial)
            cases += 1
            found += len(got)
    assert cases == 48 and found > 40


def test_vectorised_scan_grids_and_feature_rows_are_bit_identical():
    """scan_grids and the batched k feature of predict_batch equal scan_grid / k_feature per
    item bit for bit, and feature_row equals its definition on stack_arrays (ε column-major
    / 10, thickness in wavelengths, λ_ref / λ)."""
    from yellowthinfilms_b200 import learned as L
    from yellowthinfilms_b200.materials import stack_arrays
    rng = np.random.default_rng(8)
    items = [L.film_stack(rng) for _ in range(16)]
    k0s = np.array([2 * np.pi / lam for _, lam in items])
    G = L.scan_grids(k0s, 512)
    assert np.array_equal(G, np.stack([L.scan_grid(k0, 512) for k0 in k0s]))
    kf = (G / (L.K_HI * k0s)[:, None]).astype(np.float32)
    assert np.array_equal(kf, np.stack([L.k_feature(k0, L.scan_grid(k0, 512)) for k0 in k0s]))
    for st, lam in items:
        k0 = 2 * np.pi / lam
        _, _, eps, _, d = stack_arrays(st)
        ref = np.zeros(L.N_FEATURES)
        for l in range(min(len(st), L.MAX_LAYERS)):
            ref[19 * l:19 * l + 9] = eps[l].real / 10.0
            ref[19 * l + 9:19 * l + 18] = eps[l].imag / 10.0
            ref[19 * l + 18] = d[l] * k0 / (2 * np.pi)
        ref[-2] = k0 * L.LAMBDA_REF / (2 * np.pi)
        assert np.array_equal(L.feature_row(st, k0), ref.astype(np.float32))


def test_refine_levels_with_a_check_order(monkeypatch):
    """_refine_levels with check_order: the first level compares the order-8 rule with the
    same panels at the check order and returns the latter on agreement; a problem that fails
    keeps its order-8 rule and G, which the next levels halve until two levels agree. Rules and
    G are stand-ins with a known error model: G = 1 + (panel width / scale)^order."""
    from yellowthinfilms_b200 import learned as L

    def fake_gl(sets, order, ctx=None, device=False):
        # k: every panel's width repeated order times; w: the order
        out = []
        for p, _ in sets:
            p = np.asarray(p, np.float64).reshape(-1, 2)
            out.append((np.repeat(p[:, 1] - p[:, 0], order), np.full(len(p) * order, float(order))))
        return out

    def fake_G(problems, rules, ctx=None, device=False):
        return [np.array([1.0 + (k.max() / P["scale"]) ** w[0]]) for P, (k, w) in zip(problems, rules)]

    monkeypatch.setattr(L.api, "gl_rule_batch", fake_gl)
    monkeypatch.setattr(L, "batch_G", fake_G)
    panels = [np.array([[0.0, 1.0], [1.0, 2.0], [2.0, 3.0]]) for _ in range(2)]
    # easy: (1/4)^8 - (1/4)^10 < 1e-3, accepted at the check; hard: (1/1.2)^8 vs (1/1.2)^10 is not,
    # nor is halving once ((0.5/1.2)^8 against (1/1.2)^8); halving twice agrees
    probs = [dict(scale=4.0, singular=[]), dict(scale=1.2, singular=[])]
    rules = fake_gl([(p, []) for p in panels], 8)
    out, solved = [None, None], [0, 0]
    L._refine_levels(probs, range(2), rules, [p.copy() for p in panels], None, 1e-3, 4, 8, None, out, False, solved,
                     check_order=10)
    G, k, w, h, conv = out[0]
    assert conv and h == 0 and w[0] == 10 and k.max() == 1.0 and len(k) == 30
    assert solved[0] == 3 * 8 + 3 * 10
    G, k, w, h, conv = out[1]
    assert conv and h == 2 and w[0] == 8 and k.max() == 0.25 and len(k) == 12 * 8
    assert G[0] == 1.0 + (0.25 / 1.2) ** 8
    # the check level (8 + 10 nodes per panel), then the halved levels of the order-8 rule
    assert solved[1] == 3 * 8 + 3 * 10 + 6 * 8 + 12 * 8
    # without a check order the first level halves: the easy problem returns its halved rule
    rules = fake_gl([(p, []) for p in panels], 8)
    out, solved = [None, None], [0, 0]
    L._refine_levels(probs[:1], range(1), rules[:1], [panels[0].copy()], None, 1e-3, 4, 8, None, out, False, solved)
    assert out[0][4] and out[0][3] == 0 and out[0][2][0] == 8 and out[0][1].max() == 0.5 and solved[0] == 3 * 8 + 6 * 8
