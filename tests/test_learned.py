"""The learned node placement: MLP kernels against the FP64 restatement, training on
solver-generated data, and what the trained network gains over the plain fixed grid."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    from yellowthinfilms_b200 import learned
    return learned


def _random_net(L, seed=0):
    net = L.new_network(seed=seed)
    rng = np.random.default_rng(seed)
    p = net.params
    net.params = (p + rng.normal(0, 0.02, p.size)).astype(np.float32)
    return net


def test_mlp_forward_and_gradients_match_oracle(L):
    """ytf_mlp forward outputs and the backward kernels' parameter gradient against the FP64
    numpy restatement (same BF16-rounded weights): FP32 accumulation over ≤ 256-term dot
    products, so ≤ 1e-4 relative."""
    import ytf_mlp_ref as R
    net = _random_net(L, 3)
    rng = np.random.default_rng(4)
    B = 96
    X = rng.normal(0, 1, (B, L.N_FEATURES)).astype(np.float32)
    T = np.stack([rng.normal(0, 1, B), rng.uniform(0, 1, B)], 1).astype(np.float32)
    p = net.params.astype(np.float64)
    out = net.forward(X)
    _, H = R.forward(p, net.sizes, X)
    assert np.max(np.abs(out - H[-1])) <= 1e-4 * max(1.0, np.max(np.abs(H[-1])))
    loss, g = net.gradients(X, T)
    lo, go = R.loss_and_grad(p, net.sizes, X, T)
    assert abs(loss - lo) <= 1e-5 * max(1.0, abs(lo))
    assert np.linalg.norm(g - go) <= 1e-4 * np.linalg.norm(go), np.linalg.norm(g - go) / np.linalg.norm(go)
    # layer by layer too (the small last layer would hide in the global norm)
    o = 0
    for l in range(1, len(net.sizes)):
        n = net.sizes[l] * net.sizes[l - 1] + net.sizes[l]
        assert np.linalg.norm(g[o:o + n] - go[o:o + n]) <= 1e-4 * np.linalg.norm(go[o:o + n]) + 1e-12, l
        o += n


def test_mlp_training_reduces_loss(L):
    """Adam steps of libytf's kernels on a solver-generated set lower the loss (its floor is
    not 0: the logistic term on soft pole scores keeps their entropy)."""
    X, T = L.training_set(24, n_k=512, seed=5)
    net = L.new_network(seed=1)
    l0, _ = net.gradients(X[:4096], T[:4096])
    losses = L.train(net, X, T, steps=300, batch=2048, lr=1e-3)
    l1, _ = net.gradients(X[:4096], T[:4096])
    assert np.all(np.isfinite(losses))
    assert l1 < 0.6 * l0, (l0, l1)


Z_ROWS = np.linspace(0.0, 200.0, 8)  # observer heights over 0-200 nm above the film
H_MIN = 20.0 + Z_ROWS.min()          # source height + lowest observer: the shortest reflected path


def _check_fn(api, st, k0, rho_max_wl=5.0):
    lam = 2 * np.pi / k0
    rho = np.exp(np.linspace(np.log(0.01 * lam), np.log(rho_max_wl * lam), 16))

    def G(k, w):
        c = api.build_cavity_transfer_1d(st, k0, 1, k, w, obs_layers=[1])
        return api.closed_form_G(c, 1, 20.0, Z_ROWS, rho, [0.0], terms="scattered")
    return G


def plain_solved_to_agreement(L, api, st, k0, rho_max, G, max_halvings=8):
    """The plain fixed rule (point_kx_grid without the pole scan) halved until G on two
    successive levels agrees to 1e-6: (nodes solved over all levels, G of the finer level)."""
    k, w, info = api.point_kx_grid(st, k0, 1, h_min=H_MIN, rho_max=rho_max, scan=False)
    panels = info["panels"]
    sing = sorted(set(api.layer_light_lines(st[0], k0)) | set(api.layer_light_lines(st[-1], k0)))
    Gk, solved = G(k, w), len(k)
    for _ in range(max_halvings + 1):
        panels = api.halve_panels([tuple(p) for p in panels])
        k, w = api.gl_rule(panels, 8, singular=sing)
        Gh = G(k, w)
        solved += len(k)
        if np.linalg.norm(Gk - Gh) <= 1e-6 * np.linalg.norm(Gh):
            return solved, Gh
        Gk = Gh
    return solved, None


def test_learned_rule_gains_over_the_method_without_it(L):
    """What the trained network gains, at the dipole problem's observation heights (0-200 nm
    above the film, h_min = 20 nm, so the rule runs to Kcut = 25 / h_min and meets the
    films' high-k guided modes). On held-out stacks the network proposes candidate poles,
    one batched device call samples the exact response around them, fixed_kρ_rule is built on
    the result, and the acceptance check (G on the same panels at Gauss–Legendre order 10)
    accepts the rule (returning the order-10 level) or the plain method halves it until two
    levels agree. Against a converged reference (scanned rule at
    rtol 1e-10, halved):
      * every returned G is within 1e-6 (the metric's bound);
      * most proposals are accepted by the check;
      * the plain fixed rule without pole knowledge (light-line breaks, u² substitution),
        halved until two levels agree, solves more nodes in total than the learned method."""
    from yellowthinfilms_b200 import api
    X, T = L.training_set(600, n_k=1024, seed=11)
    net = L.new_network(seed=2)
    L.train(net, X, T, steps=4000, batch=4096, lr=1e-3)
    rng = np.random.default_rng(123)
    rows = []
    for _ in range(8):
        st, lam = L.film_stack(rng)
        k0 = 2 * np.pi / lam
        G = _check_fn(api, st, k0, 5.0)
        kr, wr, ir = api.point_kx_grid(st, k0, 1, h_min=H_MIN, rho_max=5 * lam, rtol=1e-10)
        Gref = G(*L.halved(st, k0, ir["panels"], 8))
        assert np.linalg.norm(G(kr, wr) - Gref) <= 1e-9 * np.linalg.norm(Gref)
        k, w, info = L.learned_rule(net, st, k0, 1, h_min=H_MIN, rho_max=5 * lam, check=G)
        err = np.linalg.norm(info["G"] - Gref) / np.linalg.norm(Gref)
        # accepted: the order-8 proposal and the returned order-10 rule on the same panels
        solved_learned = len(k) * 9 // 5 if info["learned"] else len(k) * 2
        n_plain, Gp = plain_solved_to_agreement(L, api, st, k0, 5 * lam, G)
        err_plain = np.linalg.norm(Gp - Gref) / np.linalg.norm(Gref) if Gp is not None else np.inf
        rows.append(dict(acc=bool(info["learned"]), err=err, err_plain=err_plain, n=len(k),
                         solved=solved_learned, solved_plain=n_plain))
    msg = "\n".join(str(r) for r in rows)
    assert all(r["err"] <= 1e-6 for r in rows), msg
    assert all(r["err_plain"] <= 1e-6 for r in rows), msg
    assert sum(r["acc"] for r in rows) >= 5, msg
    assert np.mean([r["solved_plain"] / r["solved"] for r in rows]) >= 1.2, msg


def test_untrained_network_falls_back_to_the_plain_method(L):
    """An untrained network proposes poles in the wrong places; the acceptance check rejects its
    rule and the plain method refines it by halving until two levels agree, so the returned G
    still meets the tolerance."""
    from yellowthinfilms_b200 import api
    net = L.new_network(seed=9)
    rng = np.random.default_rng(77)
    st, lam = L.film_stack(rng)
    k0 = 2 * np.pi / lam
    G = _check_fn(api, st, k0, 0.2)
    kr, wr, ir = api.point_kx_grid(st, k0, 1, h_min=H_MIN, rho_max=0.2 * lam, rtol=1e-10)
    Gref = G(*L.halved(st, k0, ir["panels"], 8))
    k, w, info = L.learned_rule(net, st, k0, 1, h_min=H_MIN, rho_max=0.2 * lam, check=G)
    assert np.array_equal(info["G"], G(k, w))
    assert np.linalg.norm(info["G"] - Gref) <= 1e-6 * np.linalg.norm(Gref)
    if not info["learned"]:
        assert info["halvings"] >= 1


def test_batched_rules_equal_per_stack_rules(L):
    """learned_rules_batch and plain_rules_batch (G evaluations batched over problems) give,
    problem by problem, the rules and G of learned_rule and of the per-stack plain halving,
    bit for bit (batched builds and syntheses equal single ones bit for bit)."""
    from yellowthinfilms_b200 import api
    net = _random_net(L, 7)
    rng = np.random.default_rng(31)
    probs = []
    for _ in range(3):
        st, lam = L.film_stack(rng)
        k0 = 2 * np.pi / lam
        for rw in (0.2, 5.0):
            probs.append(dict(stack=api.Stack(st), layers=st, k0=k0, source_layer=1, zsrc_local=20.0,
                              z=np.linspace(60.0, 200.0, 6), rho=np.exp(np.linspace(np.log(0.01 * lam), np.log(rw * lam), 16)),
                              terms="scattered", h_min=80.0, rho_max=rw * lam))
    outl = L.learned_rules_batch(net, probs)
    outp = L.plain_rules_batch(probs)
    for P, (gl, kl, wl, acc, h), (gp, kp, wp, hp, conv) in zip(probs, outl, outp):
        def G(k, w):
            c = api.build_cavity_transfer_1d(P["stack"], P["k0"], 1, k, w, obs_layers=[1])
            return api.closed_form_G(c, 1, 20.0, P["z"], P["rho"], [0.0], terms="scattered")
        k, w, info = L.learned_rule(net, P["stack"], P["k0"], 1, h_min=80.0, rho_max=P["rho_max"], check=G)
        assert np.array_equal(k, kl) and np.array_equal(info["G"], gl) and bool(info["learned"]) == bool(acc)
        k2, w2, inf2 = api.point_kx_grid(P["stack"], P["k0"], 1, h_min=80.0, rho_max=P["rho_max"], scan=False)
        panels, Gk = inf2["panels"], G(k2, w2)
        for _ in range(hp + 1 if conv else hp):  # a converged problem returns the finer level of its pair
            panels = api.halve_panels([tuple(p) for p in panels])
            k2, w2 = api.gl_rule(panels, 8, singular=L._sing(P))
            Gk = G(k2, w2)
        assert np.array_equal(k2, kp) and np.array_equal(Gk, gp)


def test_cavity_response_batch_equals_single_calls(L):
    """ytf_cavity_response_batch gives every item's responses bit for bit as its own
    ytf_cavity_response call (empty items included); a bad item is named in the error."""
    from yellowthinfilms_b200 import api
    rng = np.random.default_rng(17)
    items = []
    for j in range(5):
        st, lam = L.film_stack(rng)
        k0 = 2 * np.pi / lam
        n = 0 if j == 2 else int(rng.integers(1, 400))
        items.append((api.Stack(st), k0, 1, k0 * rng.uniform(0.2, 20.0, n)))
    got = api.cavity_response_batch(items)
    assert len(got) == len(items)
    for (st, k0, s, ks), R in zip(items, got):
        assert len(R) == len(ks)
        if len(ks):
            assert np.array_equal(R, api.cavity_response(st, k0, s, ks))
    bad = list(items)
    bad[3] = (items[3][0], items[3][1], 3, items[3][3])
    with pytest.raises(api.YTFError, match="item 3"):
        api.cavity_response_batch(bad)


def test_device_resident_rules_equal_host_rules(L):
    """learned_rules_batch / plain_rules_batch with G and the acceptance checks in device
    memory (the rules as CUDA tensors, straight from the device Gauss-Legendre expansion into
    the transfer build) return the same rules and, bit for bit, the same G as the host-array
    form."""
    from yellowthinfilms_b200 import api
    net = _random_net(L, 7)
    rng = np.random.default_rng(41)
    probs = []
    for _ in range(4):
        st, lam = L.film_stack(rng)
        k0 = 2 * np.pi / lam
        probs.append(dict(stack=api.Stack(st), layers=st, k0=k0, source_layer=1, zsrc_local=20.0,
                          z=np.linspace(60.0, 200.0, 12), rho=np.exp(np.linspace(np.log(0.01 * lam), np.log(5 * lam), 40)),
                          terms="scattered", h_min=80.0, rho_max=5 * lam, precision="int8x3"))
    for fn in (lambda d: L.plain_rules_batch(probs, device=d), lambda d: L.learned_rules_batch(net, probs, device=d)):
        host, dev = fn(False), fn(True)
        for a, b in zip(host, dev):
            npy = lambda x: x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)
            assert np.array_equal(a[1], npy(b[1])) and np.array_equal(a[2], npy(b[2])) and a[3:] == b[3:]
            assert np.array_equal(a[0], b[0].cpu().numpy())


def test_gl_rule_batch_equals_single_calls(L):
    """ytf_gl_rule_batch: every panel set's nodes and weights bit for bit as its own
    ytf_gl_rule call (each set with its own singular points; empty sets included)."""
    from yellowthinfilms_b200 import api
    from yellowthinfilms_b200.materials import FlatOpticalLayer, IsotropicMaterial
    rng = np.random.default_rng(5)
    sets = []
    for j in range(6):
        n = 0 if j == 3 else int(rng.integers(1, 60))
        e = np.sort(rng.uniform(0.0, 3.0, n + 1))
        P = np.stack([e[:-1], e[1:]], 1)
        sing = [float(e[0]), float(e[-1])] if j % 2 == 0 and n else []
        sets.append((P, sing))
    got = api.gl_rule_batch(sets, 8)
    for (P, sing), (k, w) in zip(sets, got):
        if len(P) == 0:
            assert len(k) == 0 and len(w) == 0
            continue
        k1, w1 = api.gl_rule(P, 8, singular=sing)
        assert np.array_equal(k, k1) and np.array_equal(w, w1)
    # the device form (ytf_gl_rule_batch_device): the same rules as CUDA tensors, and a 1D
    # transfer build from them equal to one from the host arrays
    dev = api.gl_rule_batch(sets, 8, device=True)
    for (k, w), (kd, wd) in zip(got, dev):
        assert kd.is_cuda and np.array_equal(k, kd.cpu().numpy()) and np.array_equal(w, wd.cpu().numpy())
    st = [FlatOpticalLayer(IsotropicMaterial(1.0), 0.5), FlatOpticalLayer(IsotropicMaterial(2.25), 0.3),
          FlatOpticalLayer(IsotropicMaterial(1.0), 0.5)]
    items = [dict(stack=st, omega=2.0, source_layer=1, kx_nodes=k, wt_nodes=w, obs_layers=[1]) for k, w in got if len(k)]
    items_d = [dict(stack=st, omega=2.0, source_layer=1, kx_nodes=k, wt_nodes=w, obs_layers=[1]) for k, w in dev if len(k)]
    for a, b in zip(api.build_cavity_transfer_batch(items), api.build_cavity_transfer_batch(items_d)):
        ea, eb = a.export(), b.export()
        assert all(np.array_equal(ea[x], eb[x]) for x in ea)


def test_rule_panels_batch_equals_single_calls(L):
    """ytf_rule_panels_batch (host threads): every problem's panels bit for bit as its own
    rule_panels call, with and without given poles (none, some, empty lists), and a bad
    problem named in the error."""
    from yellowthinfilms_b200 import api
    rng = np.random.default_rng(19)
    probs = []
    for j in range(40):
        st, lam = L.film_stack(rng)
        k0 = 2 * np.pi / lam
        poles = None if j % 3 == 0 else ([] if j % 3 == 1 else [(k0 * rng.uniform(1.2, 30.0), k0 * 1e-3)])
        probs.append(dict(stack=api.Stack(st), omega=k0, source_layer=1, h_min=20.0 + 5 * (j % 4),
                          rho_max=5 * lam, poles=poles))
    got = api.rule_panels_batch(probs)
    for P, g in zip(probs, got):
        ref = api.rule_panels(P["stack"], P["omega"], 1, h_min=P["h_min"], rho_max=P["rho_max"], poles=P["poles"])
        assert np.array_equal(g, ref)
    bad = list(probs)
    bad[7] = dict(probs[7], h_min=-1.0)
    with pytest.raises(api.YTFError, match="problem 7"):
        api.rule_panels_batch(bad)


def test_concurrent_shares_equal_serial_calls(L):
    """learned.concurrent_shares: two shares of problems run at once on two host threads,
    each with its own libytf context and CUDA stream, return bit for bit what the same shares
    return one after the other (device rules, int8x3 grouped synthesis, device G)."""
    import torch
    from yellowthinfilms_b200 import api
    net = _random_net(L, 11)
    rng = np.random.default_rng(53)
    ctxs = [api.Context(0), api.Context(0)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    for c, s in zip(ctxs, streams):
        c.set_stream(s.cuda_stream)
    shares = [[], []]
    for j in range(6):
        st, lam = L.film_stack(rng)
        k0 = 2 * np.pi / lam
        shares[j % 2].append(dict(stack=api.Stack(st, ctxs[j % 2]), layers=st, k0=k0, source_layer=1, zsrc_local=20.0,
                                  z=np.linspace(0.0, 200.0, 8), h_min=20.0, terms="scattered", precision="int8x3",
                                  rho=np.exp(np.linspace(np.log(0.01 * lam), np.log(5 * lam), 24)), rho_max=5 * lam))
    # the network's forward runs before the shares (one MLP object is not shared by threads)
    preds = [L.predict_batch(net, [(P["layers"], P["k0"]) for P in sh], 512) for sh in shares]
    for fn in (lambda j, c: L.plain_rules_batch(shares[j], ctx=c, device=True),
               lambda j, c: L.learned_rules_batch(net, shares[j], ctx=c, device=True, n_scan=512, pred=preds[j])):
        both = L.concurrent_shares(fn, [0, 1], ctxs, streams)
        torch.cuda.synchronize()
        for j in range(2):
            with torch.cuda.stream(streams[j]):
                one = fn(j, ctxs[j])
            torch.cuda.synchronize()
            for a, b in zip(both[j], one):
                assert torch.equal(a[0], b[0]) and len(a[1]) == len(b[1]) and a[3:] == b[3:]
