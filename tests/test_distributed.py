"""The multi-GPU partitions (yellowthinfilms_b200.distributed) on two gloo ranks on the CPU:
the k-node shard of one item summed by one all_reduce equals the whole rule's G (G is
linear in the quadrature sum, as the reference's chunked_2d uses, mod_ClosedFormGrid.jl:
449-467), and independent items spread over the ranks come back, gathered, equal to solving
them in one process. The partial sums here come from the CPU checker; on GPUs the same
partition and reduction run on the product's CUDA synthesis over NCCL."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_balanced_shares_and_node_chunks():
    from yellowthinfilms_b200.distributed import balanced_shares, node_chunk
    costs = [5, 1, 9, 3, 3, 7, 2]
    for world in (1, 2, 3, 4, 8):
        sh = balanced_shares(costs, world)
        assert sorted(i for s in sh for i in s) == list(range(len(costs)))
        assert balanced_shares(costs, world) == sh  # deterministic
        loads = [sum(costs[i] for i in s) for s in sh]
        assert max(loads) - min(loads) <= max(costs)
    assert balanced_shares(costs, 2) == [[2, 3, 4], [0, 1, 5, 6]]  # loads 15 and 15
    for n, align, world in ((64, 8, 3), (8, 8, 4), (0, 8, 2), (40, 8, 5), (13, 1, 4)):
        sl = [node_chunk(n, r, world, align) for r in range(world)]
        assert sl[0].start == 0 and sl[-1].stop == n
        for a, b in zip(sl[:-1], sl[1:]):
            assert a.stop == b.start
        assert all((s.stop - s.start) % align == 0 for s in sl)
    with pytest.raises(ValueError):
        node_chunk(10, 0, 2, 8)


def _oracle_G_julia(stack, k0, kc, wc, z, rho):
    import torch
    import ytf_oracle as oracle
    if len(kc) == 0:
        return torch.zeros(len(rho) * len(z) * 9, dtype=torch.complex128)
    c = oracle.build_cavity_transfer_1d(stack, k0, 1, kc, wc, obs_layers=[1])
    G = oracle.closed_form_G(c, 1, 20.0, z, rho, [0.0], terms="scattered")
    return torch.from_numpy(np.ascontiguousarray(G.transpose(4, 3, 2, 1, 0)).ravel())


def _problem():
    from yellowthinfilms_b200.materials import FlatOpticalLayer, IsotropicMaterial, UniaxialMaterial
    st = [FlatOpticalLayer(IsotropicMaterial(1.0), 200.0),
          FlatOpticalLayer(UniaxialMaterial(-3.0 + 0.4j, 4.0 + 0.2j), 50.0),
          FlatOpticalLayer(IsotropicMaterial(2.25), 100.0)]
    k0 = 2 * np.pi / 600.0
    import ytf_oracle as oracle
    x, w = oracle.gauss_legendre(8)
    e = np.linspace(0.0, 20 * k0, 17)
    k = (0.5 * (e[1:] + e[:-1])[:, None] + 0.5 * np.diff(e)[:, None] * x[None, :]).ravel()
    wt = (0.5 * np.diff(e)[:, None] * w[None, :]).ravel()
    return st, k0, k, wt, np.linspace(0.0, 200.0, 4), np.geomspace(6.0, 3000.0, 8)


def _rank_main(rank, world, port, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    from datetime import timedelta
    import torch.distributed as dist
    from yellowthinfilms_b200 import distributed as D
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        st, k0, k, w, z, rho = _problem()
        G = D.sharded_green(lambda kc, wc: _oracle_G_julia(st, k0, kc, wc, z, rho), k, w, order=8)
        # independent items: one rule per wavelength, gathered to rank 0
        items, greens = [], []
        for lam in (500.0, 600.0, 700.0):
            kk = 2 * np.pi / lam
            items.append(dict(stack=st, omega=kk, source_layer=1, kx_nodes=k * kk / k0, wt_nodes=w * kk / k0))
            greens.append(dict(z=z, rho=rho))
        solve = lambda tr, gr: [_oracle_G_julia(t["stack"], t["omega"], t["kx_nodes"], t["wt_nodes"], g["z"], g["rho"])
                                for t, g in zip(tr, gr)]
        out = D.spread_items(items, greens, solve=solve, gather_to=0)
        dist.barrier()
        results[rank] = (G.numpy(), out if rank == 0 else sorted(out))
    finally:
        dist.destroy_process_group()


def test_node_shard_allreduce_and_item_spread_on_two_gloo_ranks():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        res = m.dict()
        ps = [ctx.Process(target=_rank_main, args=(r, 2, port, res)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(180)
            assert p.exitcode == 0
        res = dict(res)
    st, k0, k, w, z, rho = _problem()
    whole = _oracle_G_julia(st, k0, k, w, z, rho).numpy()
    for r in (0, 1):
        G = res[r][0]
        assert np.linalg.norm(G - whole) <= 1e-12 * np.linalg.norm(whole)
    gathered = res[0][1]
    assert len(gathered) == 3
    for lam, g in zip((500.0, 600.0, 700.0), gathered):
        kk = 2 * np.pi / lam
        ref = _oracle_G_julia(st, kk, k * kk / k0, w * kk / k0, z, rho).numpy()
        assert np.array_equal(np.asarray(g), ref)
    assert res[1][1]  # rank 1 kept its own share


@pytest.mark.gpu
def test_device_partials_of_the_node_chunks_sum_to_the_whole_rule():
    """The product's partial-G callable on each rank's chunk of a rule (the ranks emulated one
    after another on one GPU, no collective): the partials sum to closed_form_G on the whole
    rule to rounding, and to the oracle."""
    import torch
    import ytf_oracle as oracle
    from yellowthinfilms_b200 import api
    from yellowthinfilms_b200 import distributed as D
    st, k0, k, w, z, rho = _problem()
    part = D.device_partial_green(st, k0, 1, 1, 20.0, z, rho, [0.0], terms="scattered")
    tot = sum(part(k[D.node_chunk(len(k), r, 3, 8)], w[D.node_chunk(len(k), r, 3, 8)]) for r in range(3))
    whole = part(k, w)
    assert float(torch.linalg.vector_norm(tot - whole) / torch.linalg.vector_norm(whole)) < 1e-13
    ref = _oracle_G_julia(st, k0, k, w, z, rho).numpy()
    assert np.linalg.norm(tot.cpu().numpy() - ref) <= 1e-10 * np.linalg.norm(ref)
    assert float(torch.linalg.vector_norm(part(k[:0], w[:0]))) == 0.0
