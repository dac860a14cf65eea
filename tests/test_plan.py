"""Uneven-batch plans (one CUDA graph per step: persistent tile-queue node-solve kernels,
batched small-set synthesis) and their autotuner. The plan's caches must equal
ytf_transfer_batch's bit for bit (the same per-unit arithmetic in persistent form), its G
must equal the per-item FP64 synthesis to rounding (the node sums run in another order) and
the oracle on the smallest items; the tuner's descent and its JSON database are checked on
the CPU with a synthetic cost."""
import json

import numpy as np
import pytest

from helpers import relerr


# ------------------------------------------------------------------ autotuner (CPU) ---

def _fake_items(n1d=3, n2d=2, nodes=1000, layers=5, pix=4):
    tr, syn = [], []
    for i in range(n1d + n2d):
        st = [None] * layers
        if i < n1d:
            tr.append(dict(stack=st, kx_nodes=np.zeros(nodes), wt_nodes=np.zeros(nodes)))
        else:
            tr.append(dict(stack=st, kr_nodes=np.zeros(nodes // 8), kr_weights=np.zeros(nodes // 8),
                           phi_nodes=np.zeros(8), phi_weights=np.zeros(8)))
        syn.append(dict(obs_layer=1, zsrc_local=0.0, z_obs=[0.0], xs=np.zeros(pix), ys=np.zeros(pix)))
    return tr, syn


def test_config_class_buckets():
    from yellowthinfilms_b200 import autotune as A
    tr, syn = _fake_items()
    c = A.config_class(tr, syn)
    assert c == "items2_nodes9_layers8_2d-some_pix4"
    tr1, syn1 = _fake_items(n1d=5, n2d=0, layers=20)
    assert A.config_class(tr1, syn1) == "items2_nodes9_layers32_2d-none_pix4"
    tr2, syn2 = _fake_items(n1d=0, n2d=4, nodes=4096, layers=12, pix=8)
    assert A.config_class(tr2, syn2) == "items2_nodes12_layers16_2d-all_pix6"


def test_descent_finds_the_separable_minimum():
    """On a separable cost the coordinate descent lands on the per-parameter minimum and
    measures each candidate at most once."""
    from yellowthinfilms_b200 import autotune as A
    target = dict(ctas_per_sm=2, block=256, tile=4096, chunk=512, synth_ctas_per_sm=4)
    calls = []

    def cost(t):
        calls.append(t)
        return sum(abs(np.log2(t[k]) - np.log2(v)) for k, v in target.items()) + 1.0

    best, ms, tried = A.descend(cost)
    assert best == target and ms == 1.0
    keys = [tuple(sorted(t.items())) for t in calls]
    assert len(keys) == len(set(keys)) == len(tried)
    assert len(calls) <= 1 + sum(len(v) for v in A.CANDIDATES.values())


def test_tune_database_roundtrip_and_reuse(tmp_path, monkeypatch):
    """tuned_plan measures and persists a new (arch, class) and reuses the record later
    without measuring (a stand-in plan class counts the runs)."""
    from yellowthinfilms_b200 import api, autotune as A
    runs = []

    class FakePlan:
        def __init__(self, tr, syn, tune=None, ctx=None):
            self.tune = dict(A.DEFAULT, **(tune or {}))

        def retune(self, t):
            self.tune = dict(t)

        def run(self):
            runs.append(dict(self.tune))

        def wait(self):
            return 10.0 / self.tune["ctas_per_sm"] + self.tune["chunk"] / 1e4

    monkeypatch.setattr(api, "BatchPlan", FakePlan)
    path = str(tmp_path / "tune.json")
    tr, syn = _fake_items()
    plan, rec = A.tuned_plan(tr, syn, arch="sm_100 test", path=path)
    assert rec["tune"]["ctas_per_sm"] == 8 and rec["tune"]["chunk"] == 512
    assert plan.tune == rec["tune"] and len(runs) > 0
    db = json.load(open(path))
    assert list(db) == ["sm_100 test|" + A.config_class(tr, syn)]
    n = len(runs)
    plan2, rec2 = A.tuned_plan(tr, syn, arch="sm_100 test", path=path)
    assert len(runs) == n and rec2 == rec and plan2.tune == rec["tune"]


# ---------------------------------------------------------------------- plans (GPU) ---

def _small_uneven(n=24):
    import bench
    tr, syn = bench.uneven_batch(n, nk_lo=64, nk_hi=2048)
    return tr, syn


@pytest.mark.gpu
def test_plan_matches_batch_and_oracle(oracle):
    """24 uneven stacks (2-24 layers, 1D and 2D rules): the plan's caches equal
    ytf_transfer_batch's bit for bit, its G equals the per-item FP64 synthesis to 1e-12 and
    the oracle on the two smallest items; two runs agree bit for bit; other tiles (persistent
    grid, block, tile, chunk) change G only by rounding."""
    from yellowthinfilms_b200 import api
    tr, syn = _small_uneven()
    plan = api.BatchPlan(tr, syn)
    info = plan.info()
    assert info["kernels"] >= 4 and info["passes"] >= 1
    G1 = [g.copy() for g in plan()]
    G1b = [g.copy() for g in plan()]
    for a, b in zip(G1, G1b):
        assert np.array_equal(a, b)
    caches = api.build_cavity_transfer_batch([dict(t, rotation=False) for t in tr])
    Gref = api.closed_form_G_batch([dict(y, cache=c) for y, c in zip(syn, caches)])
    for i, (c, g, gr) in enumerate(zip(caches, G1, Gref)):
        pc = plan.cache(i)
        e1, e2 = pc.export(), c.export()
        for key in ("T", "Qf", "Qb", "sf", "sb", "basis"):
            for x, y in zip(np.atleast_1d(e1[key]), np.atleast_1d(e2[key])):
                assert np.array_equal(x, y), (i, key)
        assert all(np.array_equal(x, y) for x, y in zip(pc.status(), c.status())), i
        assert relerr(g, gr) < 1e-12, (i, relerr(g, gr))
    small = sorted(range(len(tr)), key=lambda i: len(tr[i].get("kx_nodes", ())) or 8 * len(tr[i]["kr_nodes"]))[:2]
    for i in small:
        t, y = tr[i], syn[i]
        if "kx_nodes" in t:
            oc = oracle.build_cavity_transfer_1d(t["stack"], t["omega"], t["source_layer"], t["kx_nodes"],
                                                 t["wt_nodes"], obs_layers=t["obs_layers"])
        else:
            oc = oracle.build_cavity_transfer_2d(t["stack"], t["omega"], t["source_layer"], t["kr_nodes"],
                                                 t["kr_weights"], t["phi_nodes"], t["phi_weights"],
                                                 obs_layers=t["obs_layers"], rotation=False)
        Go = oracle.closed_form_G(oc, y["obs_layer"], y["zsrc_local"], y["z_obs"], y["xs"], y["ys"])
        assert relerr(G1[i], Go) < 1e-10, (i, relerr(G1[i], Go))
    for tune in (dict(block=256, ctas_per_sm=1, tile=256, chunk=512, synth_ctas_per_sm=1),
                 dict(block=128, ctas_per_sm=8, tile=4096, chunk=8192, synth_ctas_per_sm=4)):
        plan.retune(tune)
        G2 = plan()
        for i, (a, b) in enumerate(zip(G1, G2)):
            assert relerr(b, a) < 1e-13, (tune, i)


@pytest.mark.gpu
def test_plan_reads_updated_inputs_and_device_outputs():
    """Every run re-reads the held inputs: new z rows give closed_form_G at the new rows; an
    item whose `out` is a device tensor is written by the graph itself."""
    import torch
    from yellowthinfilms_b200 import api
    tr, syn = _small_uneven(6)
    y0 = syn[0]
    out = torch.zeros(len(y0["xs"]) * len(y0["ys"]) * len(y0["z_obs"]) * 9, dtype=torch.complex128, device="cuda:0")
    syn = [dict(syn[0], out=out)] + syn[1:]
    plan = api.BatchPlan(tr, syn)
    plan()
    z = plan.inputs(1)["z"]
    z *= 0.5
    G = plan()
    caches = api.build_cavity_transfer_batch([dict(t, rotation=False) for t in tr[:2]])
    G0 = api.closed_form_G(caches[0], y0["obs_layer"], y0["zsrc_local"], y0["z_obs"], y0["xs"], y0["ys"])
    y1 = syn[1]
    G1 = api.closed_form_G(caches[1], y1["obs_layer"], y1["zsrc_local"], z, y1["xs"], y1["ys"])
    g0 = out.cpu().numpy().reshape(3, 3, len(y0["z_obs"]), len(y0["ys"]), len(y0["xs"])).transpose(4, 3, 2, 1, 0)
    assert relerr(g0, G0) < 1e-12
    assert relerr(G[1], G1) < 1e-12


@pytest.mark.gpu
def test_plan_argument_errors():
    from yellowthinfilms_b200 import api
    tr, syn = _small_uneven(12)
    one = next(i for i, t in enumerate(tr) if "kx_nodes" in t)
    bad = list(syn)
    bad[one] = dict(syn[one], precision="int8x3")
    with pytest.raises(api.YTFError, match="plan item %d" % one):
        api.BatchPlan(tr, bad)
    bad = list(syn)
    bad[one] = dict(syn[one], xs=np.linspace(0.1, 3.0, 9) * 50, ys=np.linspace(0.2, 2.0, 9) * 50)
    with pytest.raises(api.YTFError, match="distinct radii"):
        api.BatchPlan(tr, bad)
    bad = list(syn)
    bad[one] = dict(syn[one], z_obs=np.linspace(0.1, 0.2, 9) * syn[one]["zsrc_local"])
    with pytest.raises(api.YTFError, match="z rows"):
        api.BatchPlan(tr, bad)
    p = api.BatchPlan(tr, syn)
    with pytest.raises(api.YTFError, match="multiple of 16"):
        p.retune(dict(chunk=100))
    assert len(p()) == 12  # a refused retune keeps the last graph


@pytest.mark.gpu
def test_plan_large_2d_sets_in_the_graph():
    """2D items beyond the small-set limits (32x32 pixels, 8 z rows) or in a tensor-core
    precision run closed_form_G's own kernels inside the plan's graph, from the plan's own
    workspaces: G equals ytf_green_batch's bit for bit, on pageable, page-locked and device
    outputs, over
    repeated runs and after a retune; small items of the same plan keep the batched kernel."""
    import torch
    from yellowthinfilms_b200 import api
    tr, syn = _small_uneven(10)
    two = [i for i, t in enumerate(tr) if "kr_nodes" in t]
    assert len(two) >= 3
    syn = list(syn)
    xy = np.linspace(-60.0, 60.0, 32)
    precs = ["int8x3", "fp64", "split_bf16"]
    outs = {}
    for k, i in enumerate(two[:3]):
        zs = syn[i]["zsrc_local"]
        syn[i] = dict(syn[i], xs=xy, ys=xy, z_obs=np.linspace(0.2, 1.8, 8) * zs, precision=precs[k])
    dev, pin = two[1], two[0]
    outs[dev] = torch.zeros(32 * 32 * 8 * 9, dtype=torch.complex128, device="cuda:0")
    outs[pin] = torch.zeros(32 * 32 * 8 * 9, dtype=torch.complex128, pin_memory=True)  # copied into directly
    syn[dev] = dict(syn[dev], out=outs[dev])
    syn[pin] = dict(syn[pin], out=outs[pin])
    plan = api.BatchPlan(tr, syn)
    caches = api.build_cavity_transfer_batch([dict(t, rotation=False) for t in tr])
    ref = api.closed_form_G_batch([dict({k: v for k, v in y.items() if k != "out"}, cache=c) for y, c in zip(syn, caches)])
    for rep in range(3):
        if rep == 2:
            plan.retune(dict(ctas_per_sm=2, tile=512, chunk=1024))
        G = plan()
        for i in range(len(tr)):
            if i in (dev, pin):
                g = outs[i].cpu().numpy().reshape(3, 3, 8, 32, 32).transpose(4, 3, 2, 1, 0)
            else:
                g = G[i]
            if i in two[:3]:
                assert np.array_equal(g, ref[i]), (rep, i)
            else:
                assert relerr(g, ref[i]) < 1e-12, (rep, i)


@pytest.mark.gpu
def test_tuned_plan_persists_choice(tmp_path):
    from yellowthinfilms_b200 import autotune as A
    tr, syn = _small_uneven(8)
    path = str(tmp_path / "tune.json")
    plan, rec = A.tuned_plan(tr, syn, path=path, reps=1)
    assert rec["measured"] >= 5 and rec["ms"] > 0
    assert plan.tune == rec["tune"]
    plan2, rec2 = A.tuned_plan(tr, syn, path=path)
    assert rec2 == rec and plan2.tune == rec["tune"]
