"""The path on several GPUs: one process per GPU, torch.distributed for the plumbing.

The reference runs on one host and parallelises with threads over work that is independent
or linear (no counterpart of this module): its cache builds thread over k-nodes
(mod_CavityTransfer.jl:224, :362), and `chunked_2d` (mod_ClosedFormGrid.jl:449-467) builds
caches on consecutive chunks of the kρ rule and SUMS `closed_form_G` over them, which is
exact because G is linear in the quadrature sum. The two partitions here follow from that:

(i) independent items (stacks, wavelengths, source depths, observation sets): every rank
    takes a share of the items and solves them with the batched calls; no collective on the
    data path. ``spread_items`` balances the shares by node count and, on request, gathers
    every item's G to one rank afterwards.
(ii) one item whose rule is too large for one GPU (or too slow): every rank solves a
    contiguous, panel-aligned chunk of the nodes and synthesises a partial G; ONE
    all_reduce (sum) over the ranks gives every rank the whole G (``sharded_green``). Over
    NCCL the partial G stays in device memory and the sum runs over NVLink; complex values
    travel as pairs of float64.

Every rank takes the same collective calls in the same order. The synthesis itself is a
callable, so the partition and the reduction are the same code whatever computes the
partial sums (the product's CUDA path, or a CPU checker in the tests).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import numpy as np


def balanced_shares(costs: Sequence[float], world: int) -> List[List[int]]:
    """Item indices per rank: longest item first onto the least-loaded rank (ties to the lower
    rank), each share in increasing item order. Deterministic, so every rank computes the
    same partition without communication."""
    if world < 1:
        raise ValueError("balanced_shares: world must be ≥ 1")
    load = [0.0] * world
    shares: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda j: (-float(costs[j]), j)):
        r = min(range(world), key=lambda q: (load[q], q))
        shares[r].append(i)
        load[r] += float(costs[i])
    return [sorted(s) for s in shares]


def node_chunk(n: int, rank: int, world: int, align: int = 1) -> slice:
    """The contiguous slice of n rule nodes that rank owns: whole groups of ``align`` nodes
    (the panel's order, so no Gauss–Legendre panel is split), groups spread as evenly as
    possible, lower ranks first. The slices of all ranks tile range(n) in order."""
    if align < 1 or n % align:
        raise ValueError(f"node_chunk: {n} nodes are not whole groups of {align}")
    groups = n // align
    base, extra = divmod(groups, world)
    g0 = rank * base + min(rank, extra)
    g1 = g0 + base + (1 if rank < extra else 0)
    return slice(g0 * align, g1 * align)


def _world(group):
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def allreduce_sum(partial, group=None):
    """Sum a partial G over the ranks in place (one all_reduce). Complex tensors are reduced
    as their float64 (re, im) pairs, which NCCL and gloo both sum. Returns the tensor."""
    import torch
    import torch.distributed as dist
    if _world(group)[1] == 1:
        return partial
    t = torch.view_as_real(partial) if partial.is_complex() else partial
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return partial


def sharded_green(partial_G: Callable[[np.ndarray, np.ndarray], "object"], k: np.ndarray, w: np.ndarray,
                  order: int = 8, group=None):
    """G of one item whose rule (k, w) is spread over the ranks: this rank's contiguous,
    panel-aligned chunk goes to ``partial_G(k_chunk, w_chunk)`` (a torch tensor: the partial
    G of those nodes, on this rank's device for NCCL, on the CPU for gloo), then one
    all_reduce sums the partials. An empty chunk contributes zeros of the same shape, which
    ``partial_G`` must return for empty inputs. Every rank returns the whole G."""
    k, w = np.asarray(k), np.asarray(w)
    if len(k) != len(w):
        raise ValueError("sharded_green: nodes/weights length mismatch")
    rank, world = _world(group)
    sl = node_chunk(len(k), rank, world, order if len(k) % order == 0 else 1)
    return allreduce_sum(partial_G(k[sl], w[sl]), group)


def device_partial_green(stack, omega: float, source_layer: int, obs_layer: int, zsrc_local: float, z_obs, xs, ys,
                         terms: str = "all", precision: str = "fp64", ctx=None):
    """The product's partial-G callable for ``sharded_green``: a 1D cache on the node chunk
    and closed_form_G into a CUDA tensor (Julia layout, complex128)."""
    import torch
    from . import api
    nz, nx, ny = len(np.atleast_1d(z_obs)), len(np.atleast_1d(xs)), len(np.atleast_1d(ys))

    def partial(kc, wc):
        dev = (ctx or api.default_context()).device
        out = torch.zeros(nx * ny * nz * 9, dtype=torch.complex128, device=f"cuda:{dev}")
        if len(kc) == 0:
            return out
        c = api.build_cavity_transfer_1d(stack, omega, source_layer, kc, wc, obs_layers=[obs_layer], ctx=ctx)
        api.closed_form_G(c, obs_layer, zsrc_local, z_obs, xs, ys, terms=terms, precision=precision, out=out)
        return out
    return partial


def spread_items(transfer_items: Sequence[dict], green_items: Sequence[dict],
                 solve: Optional[Callable[[List[dict], List[dict]], list]] = None, gather_to: Optional[int] = 0,
                 group=None):
    """Independent items over the ranks: this rank solves its balanced share (by node
    count) with ``solve(transfer_items, green_items) -> [G]`` (default: one batched build and
    one batched synthesis through the product's calls) and no collective touches the data
    path. With ``gather_to`` set, every item's G (as numpy) is gathered to that rank
    afterwards, which returns the full list in item order; the other ranks return a dict
    {item index: G} of their own share. ``gather_to=None`` skips the gather."""
    import torch.distributed as dist
    rank, world = _world(group)
    costs = [len(t["kx_nodes"] if "kx_nodes" in t else t["kr_nodes"]) * (len(t["phi_nodes"]) if "phi_nodes" in t else 1)
             for t in transfer_items]
    mine = balanced_shares(costs, world)[rank]
    if solve is None:
        solve = _solve_batched
    got = solve([transfer_items[i] for i in mine], [green_items[i] for i in mine]) if mine else []
    own = {i: (g.cpu().numpy() if hasattr(g, "cpu") else np.asarray(g)) for i, g in zip(mine, got)}
    if gather_to is None or world == 1:
        return [own[i] for i in range(len(transfer_items))] if world == 1 else own
    parts = [None] * world if rank == gather_to else None
    dist.gather_object(own, parts, dst=gather_to, group=group)
    if rank != gather_to:
        return own
    allg = {}
    for p in parts:
        allg.update(p)
    return [allg[i] for i in range(len(transfer_items))]


def _solve_batched(transfer_items, green_items):
    from . import api
    caches = api.build_cavity_transfer_batch(transfer_items)
    return api.closed_form_G_batch([dict(g, cache=c) for g, c in zip(green_items, caches)])
