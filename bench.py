#!/usr/bin/env python
"""G(ρ, z, z') entries/s on B200 at ≤1e-6 relative error: learned-adaptive vs plain quadrature.

Default workload (`--workload learned`, the headline metric; seeded synthetic data): 4096
held-out air / uniaxial film / substrate stacks (film εo = -U[1, 6] + i 10^U[-2.5, -0.3],
εe = U[2, 6] + i 10^U[-2.7, -0.5], d U[20, 100] nm; substrate ε U[1.5, 4]; λ U[450, 750] nm),
a vertical dipole 20 nm above the film, G on 256 radii log-spaced over 0.01-5 λ x 64 heights
uniform over 0-200 nm x 9 components (scattered term). A step is one chunk of 256 stacks,
each taken to a G accurate to 1e-6 by the learned method (the node-placement MLP, trained on
1e7 solver samples before the timed region) and, timed beside it, by the plain fixed rule
halved until two levels agree. `value`: the learned method with G left in HBM; `e2e`: the
same with every G copied to page-locked host memory inside the timed region.

Other workloads: `gyro32` (the batched 8-layer biaxial/gyrotropic solve at 32 wavelengths x
65536 (kρ, φ) nodes, full 3x3 G), `uneven` (1024 uneven stacks as one CUDA graph), `bessel`
(the 1D synthesis at 4096 radii x 65536 nodes x 256 heights), `contour` (the deformed-contour
path of the 3-layer dipole problem).

The CPU baseline and `--impl reference` run the FP64 oracle (the C++ restatement of the
reference; the reference itself is Julia and cannot run here) on all host threads, on whole
units of the same workload (a held-out stack, or a whole wavelength), with no scaling.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_LAYERS = 8
N_LAMBDA = 32
N_PANELS, ORDER, N_PHI = 128, 8, 64
SRC = 4
NZ, NXY = 8, 32
SEED = 2026


def make_stack(seed=SEED):
    from yellowthinfilms_b200.materials import BiaxialMaterial, FlatOpticalLayer, GyrotropicMaterial
    rng = np.random.default_rng(seed)
    d = rng.uniform(10.0, 200.0, N_LAYERS)
    gyro = set(int(i) for i in rng.choice(N_LAYERS, N_LAYERS // 2, replace=False))
    layers = []
    for l in range(N_LAYERS):
        diag = rng.uniform(-6.0, 6.0, 3) + 1j * rng.uniform(0.01, 1.0, 3)
        if l in gyro:
            g = rng.uniform(0.0, 1.5)
            eps = np.diag(diag).astype(np.complex128)
            eps[0, 1], eps[1, 0] = 1j * g, -1j * g
            layers.append(FlatOpticalLayer(GyrotropicMaterial(eps), d[l]))
        else:
            layers.append(FlatOpticalLayer(BiaxialMaterial(*diag), d[l]))
    return layers


def uneven_batch(n_stacks=1024, seed=SEED, nk_lo=1024, nk_hi=32768):
    """The uneven-batch workload: n_stacks seeded stacks, 2-24 layers each (half-spaces
    isotropic dielectrics; interior layers isotropic, uniaxial-hyperbolic (sign Re εo ≠ sign
    Re εe) or gyrotropic; d U[5, 300] nm), λ U[450, 750] nm, source in a random layer above
    the last, observed in the source layer. Node counts log-uniform in [nk_lo, nk_hi]: a 1D
    (kx) rule for azimuthally symmetric stacks, a 2D (kρ, 8 φ) rule for gyrotropic ones, GL-8
    panels on [0, 20 k0]. Returns (transfer items, synthesis items without caches)."""
    from yellowthinfilms_b200.materials import FlatOpticalLayer, GyrotropicMaterial, IsotropicMaterial, UniaxialMaterial
    rng = np.random.default_rng(seed + 4)
    tr, syn = [], []
    for _ in range(n_stacks):
        nl = int(rng.integers(2, 25))
        layers, gyro = [], False
        for l in range(nl):
            d = float(rng.uniform(5.0, 300.0))
            kind = 0 if l in (0, nl - 1) else int(rng.integers(0, 3))
            if kind == 0:
                lo, hi = (1.0, 2.5) if l in (0, nl - 1) else (1.0, 6.0)
                m = IsotropicMaterial(complex(rng.uniform(lo, hi), rng.uniform(0.001, 0.3)))
            elif kind == 1:
                eo = complex(-rng.uniform(1.0, 6.0), rng.uniform(0.01, 0.5))
                ee = complex(rng.uniform(1.0, 6.0), rng.uniform(0.01, 0.5))
                if rng.random() < 0.5:
                    eo, ee = -eo.real + 1j * eo.imag, -ee.real + 1j * ee.imag
                m = UniaxialMaterial(eo, ee)
            else:
                g = rng.uniform(0.0, 1.5)
                eps = np.diag(rng.uniform(1.0, 6.0, 3) + 1j * rng.uniform(0.01, 0.5, 3)).astype(np.complex128)
                eps[0, 1], eps[1, 0] = 1j * g, -1j * g
                m = GyrotropicMaterial(eps)
                gyro = True
            layers.append(FlatOpticalLayer(m, d))
        lam = float(rng.uniform(450.0, 750.0))
        k0 = 2 * np.pi / lam
        src = int(rng.integers(1, nl))
        nk = int(np.exp(rng.uniform(np.log(nk_lo), np.log(nk_hi))))
        from yellowthinfilms_b200.api import gausslegendre
        xg, wg = gausslegendre(ORDER)
        nkr = max(ORDER, (nk // 8 if gyro else nk) // ORDER * ORDER)
        npan = nkr // ORDER
        edges = np.linspace(0.0, 20.0 * k0, npan + 1)
        h = 0.5 * np.diff(edges)
        kr = (0.5 * (edges[1:] + edges[:-1])[:, None] + h[:, None] * xg[None, :]).ravel()
        wr = (h[:, None] * wg[None, :]).ravel()
        ds = layers[src - 1].d
        item = dict(stack=layers, omega=k0, source_layer=src, obs_layers=[src])
        if gyro:
            item.update(kr_nodes=kr, kr_weights=wr, phi_nodes=2 * np.pi * np.arange(8) / 8,
                        phi_weights=np.full(8, 2 * np.pi / 8), rotation=False)
        else:
            item.update(kx_nodes=kr, wt_nodes=wr)
        tr.append(item)
        xy = np.linspace(-0.2 * lam, 0.2 * lam, 4)
        syn.append(dict(obs_layer=src, zsrc_local=0.5 * ds, z_obs=np.linspace(0.1 * ds, 0.9 * ds, 4), xs=xy, ys=xy))
    return tr, syn


def grids(lam, kr_stride=1, phi_take=None, gausslegendre=None):
    """(ω, kρ, wρ, φ, wφ) for one wavelength (nm units). ``gausslegendre``: the rule's
    source (libytf's by default; the CPU arms pass the oracle's, bit for bit the same)."""
    if gausslegendre is None:
        from yellowthinfilms_b200.api import gausslegendre
    k0 = 2 * np.pi / lam
    x, w = gausslegendre(ORDER)
    edges = np.linspace(0.0, 20.0 * k0, N_PANELS + 1)
    a, b = edges[:-1, None], edges[1:, None]
    kr = (0.5 * (a + b) + 0.5 * (b - a) * x[None, :]).ravel()
    wr = (0.5 * (b - a) * w[None, :]).ravel()
    phi = 2 * np.pi * np.arange(N_PHI) / N_PHI
    wphi = np.full(N_PHI, 2 * np.pi / N_PHI)
    if kr_stride > 1:
        kr, wr = kr[::kr_stride], wr[::kr_stride] * kr_stride
    if phi_take is not None:
        step = N_PHI // phi_take
        phi, wphi = phi[::step], wphi[::step] * step
    return k0, kr, wr, phi, wphi


def obs_set(stack, lam):
    d4 = stack[SRC - 1].d
    zsrc = 0.5 * d4
    zo = np.linspace(0.05 * d4, 0.95 * d4, NZ)
    xy = np.linspace(-0.2 * lam, 0.2 * lam, NXY)
    return zsrc, zo, xy, xy


ENTRIES_PER_LAMBDA = NXY * NXY * NZ * 9


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        import threading
        self.lines, self.first = [], threading.Event()
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return self

        def read():
            for line in self.proc.stdout:
                self.lines.append(line)
                self.first.set()
            self.first.set()
        self.reader = threading.Thread(target=read, daemon=True)
        self.reader.start()
        # the sampler's start-up (NVML initialisation) ends before the timed region begins
        self.first.wait(10.0)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
            self.reader.join(5.0)
            self.out = "".join(self.lines)

    def summary(self):
        rows = [r.split(",") for r in (self.out or "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][2]), "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------------------
# CPU arm: the oracle
# --------------------------------------------------------------------------------------
def cpu_sample(stack, lam):
    """Oracle on one whole wavelength (65536 nodes, 73,728 entries); returns seconds. The
    Gauss-Legendre rule is the oracle's, so no product library is loaded."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ytf_oracle as oracle
    k0, kr, wr, phi, wphi = grids(lam, gausslegendre=oracle.gauss_legendre)
    zsrc, zo, xs, ys = obs_set(stack, lam)
    t = time.perf_counter()
    c = oracle.build_cavity_transfer_2d(stack, k0, SRC, kr, wr, phi, wphi, obs_layers=[SRC], rotation=False)
    oracle.closed_form_G(c, SRC, zsrc, zo, xs, ys)
    return time.perf_counter() - t


# --------------------------------------------------------------------------------------
# ranks (one process per GPU under torchrun): every rank takes the same collective steps in
# the same order; no data-path collective, only the timing's barrier and max
# --------------------------------------------------------------------------------------
def rank_env():
    """(rank, world size, local rank) from the torchrun environment (1 process: 0, 1, 0)."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(ms, dist=None, device="cpu"):
    """The largest per-rank time: every rank calls it once per timed quantity, in order."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, ms):
    """Whole-job throughput of a weak-scaling run: every rank processes units_per_rank in
    (at most) ms milliseconds."""
    return world * units_per_rank / (ms * 1e-3)


def run_reference(args):
    """The reference arm of the gyro32 workload: one whole wavelength per step through the
    oracle (no product library in this process)."""
    rank = rank_env()[0]
    if rank != 0:  # the reference arm runs on rank 0's host cores only
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ytf_oracle as oracle
    oracle.set_threads(os.cpu_count() or 1)
    stack = make_stack()
    lams = np.linspace(450.0, 750.0, N_LAMBDA)
    for i in range(args.warmup):
        cpu_sample(stack, lams[i % N_LAMBDA])
    ts = [cpu_sample(stack, lams[(args.warmup + i) % N_LAMBDA]) for i in range(args.steps)]
    t = float(np.sum(ts))
    value = args.steps * ENTRIES_PER_LAMBDA / t
    line = {"metric": METRIC, "value": value, "unit": "entries/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded)", "impl": "reference",
            "config": dict(CONFIG, precision="fp64 (CPU oracle)"),
            "cpu_baseline": {"value": value, "unit": "entries/s", "cores": oracle.num_threads(), "kind": "port",
                             "sample": f"one whole wavelength per step ({N_PANELS * ORDER * N_PHI} nodes, "
                                       f"{ENTRIES_PER_LAMBDA} entries), timed whole; a step of the GPU arm is all "
                                       f"{N_LAMBDA} wavelengths"},
            "e2e": {"value": value, "unit": "entries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


METRIC = "G(ρ,z,z') entries/s at ≤1e-6 rel err vs the FP64 oracle (plain fixed grid), 1 B200"
CONFIG = {"workload": "batched spectral solve + full 3x3 G: 8-layer biaxial/gyrotropic stack, 32 wavelengths "
                      "450-750 nm x 65536 (kρ,φ) nodes, 8 z rows x 32x32 lateral offsets (±0.2λ)",
          "layers": N_LAYERS, "wavelengths": N_LAMBDA, "nodes_per_wavelength": N_PANELS * ORDER * N_PHI,
          "entries_per_step": ENTRIES_PER_LAMBDA * N_LAMBDA, "source_layer": SRC, "obs_layers": [SRC],
          "l2": "per-wavelength working set (node scratch ~0.6 GB) larger than L2", "seed": SEED}


# --------------------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------------------
# DRAM bytes (read + write) per launch from one ncu capture of the kernel on this workload;
# absent until captured
TRAFFIC = {"k_lateral": 81.7e6}
DTYPE = {"int8x3": "f64 solve, int8 x3-digit tensor-core synthesis (exact int32 accum)",
         "split_bf16": "f64 solve, split-bf16 x3 tensor-core synthesis (fp32 accum)",
         "fp64": "f64"}


def measured_peaks():
    """Denominators: MEASURED_PEAKS.json of this pool, else the stated fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        m = json.load(open(path))
        return {"bf16_sustained": (float(m["bf16_tflops_sustained"]), "measured (MEASURED_PEAKS.json, sustained bf16)"),
                "bf16_burst": (float(m["bf16_tflops"]), "measured (MEASURED_PEAKS.json, burst bf16)"),
                "hbm": (float(m["hbm_gbs"]), "measured (MEASURED_PEAKS.json)")}
    except (OSError, KeyError, ValueError):
        return {"bf16_sustained": (1400.0, "fallback (sustained bf16 on this pool)"),
                "bf16_burst": (1590.0, "fallback"), "hbm": (6650.0, "fallback")}


# FP64 operations per node of the per-node solve kernels on this workload, from one ncu count
# of their DFMA/DADD/DMUL instructions (2 per DFMA); absent until captured
FP64_OPS_PER_NODE = {"k_iface": 8.99e3,  # 1.79e8 DFMA + 0.97e8 DADD + 1.33e8 DMUL per 65536 nodes
                     "k_scan": 7.43e3,  # 1.59e8 DFMA + 0.57e8 DADD + 1.12e8 DMUL per 65536 nodes
                     "k_layer_modes": 9.46e3,  # 1.98e8 DFMA + 0.59e8 DADD + 1.64e8 DMUL (8 layers)
                     "k_strengths2d": 8.04e3}  # k_reflect2d + k_strengths_rows (8 z rows)  # 1.832e8 DFMA + 0.596e8 DADD + 1.009e8 DMUL (8 z rows)
FP64_NOMINAL = 37.2  # TFLOP/s: 148 SM x 64 FP64 FMA/clk x 2 x 1.965 GHz (no measured FP64 peak)


def roofline(name, prof, steps=1):
    """Roofline entry of one kernel from its CUDA-event time in the timed region; every
    step covers N_LAMBDA x 65536 nodes, in one launch per kernel (batched calls) or one per
    wavelength."""
    roof = {"kernel": name, "bound": None, "achieved": None, "peak": None, "unit": None, "frac": None,
            "traffic": TRAFFIC.get(name)}
    if name is None or name not in prof or not prof[name][1]:
        return roof
    tot_ms, nl = prof[name]
    t = tot_ms / nl * 1e-3  # seconds per launch
    nodes = N_PANELS * ORDER * N_PHI * N_LAMBDA * steps // nl  # nodes per launch
    cmacs = float(NXY * NXY * nodes * NZ * 9)  # complex multiply-adds of one lateral contraction
    work = f"8 flop per complex multiply-add x 1024 pixels x {nodes} nodes x 72 columns per launch"
    peaks = measured_peaks()
    if name in ("k_lateral_tc", "k_lateral_i8"):
        achieved = 8.0 * cmacs / t / 1e12
        peak, src = peaks["bf16_sustained"]
        roof.update(bound="tensor", achieved=achieved, peak=peak, unit="TFLOP/s", frac=achieved / peak,
                    peak_source=src, work=work)
        if name == "k_lateral_tc":
            roof.update(split_multiplier=6, tensor_flops_executed_per_launch=6 * 8.0 * cmacs)
        else:
            # six int8 digit products; int8 runs at twice the bf16 rate (nominal 4.5 vs 2.25 PFLOP/s)
            ex = 6 * 8.0 * cmacs
            roof.update(split_multiplier=6, int8_ops_executed_per_launch=ex,
                        executed_frac_of_int8_peak=ex / t / 1e12 / (2 * peak),
                        int8_peak_note="int8 peak taken as 2 x the measured bf16 figure (nominal ratio)")
    elif name == "k_lateral":
        achieved = 8.0 * cmacs / t / 1e12
        roof.update(bound="fp64", achieved=achieved, peak=FP64_NOMINAL, unit="TFLOP/s", frac=achieved / FP64_NOMINAL,
                    peak_source="nominal FP64; no measured FP64 peak", work=work)
    elif FP64_OPS_PER_NODE.get(name):
        achieved = FP64_OPS_PER_NODE[name] * nodes / t / 1e12
        roof.update(bound="fp64", achieved=achieved, peak=FP64_NOMINAL, unit="TFLOP/s",
                    frac=achieved / FP64_NOMINAL, peak_source="nominal FP64; no measured FP64 peak",
                    work=f"{FP64_OPS_PER_NODE[name]:.0f} FP64 ops per node x {nodes} nodes per launch (ncu count)")
    return roof


def run_ours(args):
    import torch
    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from yellowthinfilms_b200 import api

    ctx = api.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    stack = api.Stack(make_stack(), ctx)
    lams = np.linspace(450.0, 750.0, N_LAMBDA)
    per = [(grids(l), obs_set(stack.layers, l)) for l in lams]
    G_dev = torch.empty((N_LAMBDA, ENTRIES_PER_LAMBDA), dtype=torch.complex128, device=f"cuda:{local}")
    G_host = torch.empty((N_LAMBDA, ENTRIES_PER_LAMBDA), dtype=torch.complex128, pin_memory=True)

    transfer_items = [dict(stack=stack, omega=k0, source_layer=SRC, kr_nodes=kr, kr_weights=wr, phi_nodes=phi,
                           phi_weights=wphi, obs_layers=[SRC], rotation=False) for (k0, kr, wr, phi, wphi), _ in per]
    plans = {}

    def plan_for(host_out):
        # one CUDA graph per step: node upload, persistent node solve, the int8 tensor-core
        # synthesis of every wavelength, G into the device or the page-locked host array
        if host_out not in plans:
            from yellowthinfilms_b200 import autotune
            green = [dict(obs_layer=SRC, zsrc_local=zsrc, z_obs=zo, xs=xs, ys=ys, precision=args.precision,
                          out=(G_host[i] if host_out else G_dev[i])) for i, (_, (zsrc, zo, xs, ys)) in enumerate(per)]
            plans[host_out] = autotune.tuned_plan(transfer_items, green, ctx=ctx, reps=1)[0]
        return plans[host_out]

    def step(host_out, calls=None):
        calls = calls or args.calls
        if calls == "plan":
            p = plan_for(host_out)
            p.run()
            p.wait()
            return
        if calls == "per-call":  # one build_cavity_transfer_2d + closed_form_G call per wavelength
            for i, ((k0, kr, wr, phi, wphi), (zsrc, zo, xs, ys)) in enumerate(per):
                c = api.build_cavity_transfer_2d(stack, k0, SRC, kr, wr, phi, wphi, obs_layers=[SRC], rotation=False)
                api.closed_form_G(c, SRC, zsrc, zo, xs, ys, precision=args.precision,
                                  out=(G_host[i] if host_out else G_dev[i]))
                del c
            return
        # all wavelengths in one batched build and one batched synthesis
        caches = api.build_cavity_transfer_batch(
            [dict(stack=stack, omega=k0, source_layer=SRC, kr_nodes=kr, kr_weights=wr, phi_nodes=phi,
                  phi_weights=wphi, obs_layers=[SRC], rotation=False) for (k0, kr, wr, phi, wphi), _ in per])
        api.closed_form_G_batch(
            [dict(cache=c, obs_layer=SRC, zsrc_local=zsrc, z_obs=zo, xs=xs, ys=ys, precision=args.precision,
                  out=(G_host[i] if host_out else G_dev[i])) for i, (c, (_, (zsrc, zo, xs, ys))) in
             enumerate(zip(caches, per))])
        del caches

    def timed(host_out, profile, calls=None):
        for _ in range(args.warmup):
            step(host_out, calls)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        ctx.profile(True if profile else False)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with Clocks(local) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                step(host_out, calls)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        prof = ctx.profile_read()
        ms = max_over_ranks(ms, dist, f"cuda:{local}")
        return ms, prof, clk.summary()

    # value and e2e without the per-kernel events; the kernel split from a third, profiled pass
    # (through the batched calls when the step is a plan: the same kernels, each bracketed
    # by CUDA events, which a graph's kernels are not)
    ms, prof_plain, clocks = timed(False, False)
    ms_e2e, _, _ = timed(True, False)
    _, prof, _ = timed(False, True, "batched" if args.calls == "plan" else None)
    entries = ENTRIES_PER_LAMBDA * N_LAMBDA
    value = job_rate(entries, world, ms)
    e2e = job_rate(entries, world, ms_e2e)
    h2d = sum(8 * (len(g[1]) * 2 + len(g[3]) * 2) + 8 * (len(o[1]) + len(o[2]) + len(o[3])) for g, o in per)
    d2h = entries * 16

    # parity inside the run: first wavelength, φ subsample, GPU vs oracle on identical nodes
    err = None
    cpu = None
    if rank == 0 and not args.no_check:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ytf_oracle as oracle
        oracle.set_threads(os.cpu_count() or 1)
        k0, kr, wr, phi, wphi = grids(lams[0], phi_take=4)
        zsrc, zo, xs, ys = obs_set(stack.layers, lams[0])
        c = api.build_cavity_transfer_2d(stack, k0, SRC, kr, wr, phi, wphi, obs_layers=[SRC], rotation=False)
        G = api.closed_form_G(c, SRC, zsrc, zo, xs, ys, precision=args.precision)
        oc = oracle.build_cavity_transfer_2d(stack.layers, k0, SRC, kr, wr, phi, wphi, obs_layers=[SRC], rotation=False)
        Go = oracle.closed_form_G(oc, SRC, zsrc, zo, xs, ys)
        err = float(np.linalg.norm(G - Go) / np.linalg.norm(Go))
        dt = cpu_sample(stack.layers, lams[0])
        cpu = {"value": ENTRIES_PER_LAMBDA / dt, "unit": "entries/s", "cores": oracle.num_threads(),
               "kind": "port", "sample": f"one whole wavelength ({N_PANELS * ORDER * N_PHI} nodes, "
                                         f"{ENTRIES_PER_LAMBDA} entries), timed whole"}

    # roofline of the dominant kernel (and of the lateral contraction), from the CUDA-event
    # profile of the timed region
    top = max(prof.items(), key=lambda kv: kv[1][0])[0] if prof else None
    lateral = next((k for k in ("k_lateral_i8", "k_lateral_tc", "k_lateral") if k in prof), None)
    roof = roofline(top, prof, args.steps)
    if lateral and lateral != top:
        roof["lateral"] = roofline(lateral, prof, args.steps)
    if "k_scan" in prof and top != "k_scan":
        roof["solve"] = roofline("k_scan", prof, args.steps)
    launches = int(sum(v[1] for v in prof_plain.values()))  # the timed region's own launches
    line = {"metric": METRIC, "value": value, "unit": "entries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE[args.precision],
            "data": "synthetic (seeded)", "config": dict(CONFIG, precision=args.precision, calls={"plan": "one CUDA graph per step (ytf_plan_run + ytf_plan_wait; tuned tiles)", "batched": "batched (32 wavelengths per call)", "per-call": "per wavelength"}[args.calls]), "max_rel_err_vs_oracle": err,
            "e2e": {"value": e2e, "unit": "entries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": ms_e2e},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
            "kernels_ms_per_step_batched_pass": {k: round(v[0] / args.steps, 4) for k, v in sorted(prof.items())},
            "kernels_note": "per-kernel CUDA-event times of a separate profiled pass through the batched calls "
                            "(ytf_transfer_batch + ytf_green_batch), not of the timed graph; their sum exceeds "
                            "ms_per_step by the host work between those calls"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_uneven(args):
    """The uneven-batch workload as one autotuned plan (BatchPlan: the whole step is one CUDA
    graph: upload, persistent node-solve kernels, batched synthesis, download), one GPU. The
    tuning (coordinate descent over the plan's tiles, persisted per (GPU, batch class)) runs
    before the timed region; the per-item call path (ytf_transfer_batch + ytf_green_batch) is
    timed beside it for one step."""
    import torch
    from yellowthinfilms_b200 import api, autotune
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    tr, syn = uneven_batch()
    stacks = [api.Stack(t["stack"], ctx) for t in tr]
    items = [dict(t, stack=s) for t, s in zip(tr, stacks)]
    t0 = time.perf_counter()
    plan, rec = autotune.tuned_plan(items, syn, ctx=ctx, force=args.retune, reps=1)
    tune_s = time.perf_counter() - t0
    info = plan.info()
    for _ in range(args.warmup):
        plan.run()
        plan.wait()
    ctx.profile(True)
    dev = []
    with Clocks(0) as clk:
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for _ in range(args.steps):
            plan.run()
            dev.append(plan.wait())
        wall_ms = (time.perf_counter() - w0) * 1e3 / max(args.steps, 1)
    prof = ctx.profile_read()
    ms = float(np.mean(dev)) if dev else 0.0
    G = plan.results()
    entries = sum(g.size for g in G)
    nodes = info["nodes"]
    # the per-item call path, one step after one warm-up
    prec = "fp64"

    def calls_step():
        caches = api.build_cavity_transfer_batch([dict(t, rotation=False) for t in items], ctx=ctx)
        return api.closed_form_G_batch([dict(y, cache=c, precision=prec) for y, c in zip(syn, caches)])

    calls_step()
    torch.cuda.synchronize()
    c0 = time.perf_counter()
    Gc = calls_step()
    torch.cuda.synchronize()
    calls_ms = (time.perf_counter() - c0) * 1e3
    err_calls = max(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)) for a, b in zip(G, Gc))
    err = None
    if not args.no_check:  # two items against the oracle on identical nodes
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ytf_oracle as oracle
        oracle.set_threads(os.cpu_count() or 1)
        errs = []
        small = sorted(range(len(tr)), key=lambda i: len(tr[i].get("kx_nodes", ())) or 8 * len(tr[i]["kr_nodes"]))[:2]
        for i in small:
            t = tr[i]
            if "kx_nodes" in t:
                oc = oracle.build_cavity_transfer_1d(t["stack"], t["omega"], t["source_layer"], t["kx_nodes"],
                                                     t["wt_nodes"], obs_layers=t["obs_layers"])
            else:
                oc = oracle.build_cavity_transfer_2d(t["stack"], t["omega"], t["source_layer"], t["kr_nodes"],
                                                     t["kr_weights"], t["phi_nodes"], t["phi_weights"],
                                                     obs_layers=t["obs_layers"], rotation=False)
            y = syn[i]
            Go = oracle.closed_form_G(oc, y["obs_layer"], y["zsrc_local"], y["z_obs"], y["xs"], y["ys"])
            errs.append(float(np.linalg.norm(G[i] - Go) / np.linalg.norm(Go)))
        err = max(errs)
    line = {"metric": METRIC, "value": args.steps and entries / (ms * 1e-3), "unit": "entries/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[prec], "data": "synthetic (seeded)",
            "config": {"workload": "uneven batch: 1024 stacks, 2-24 layers (isotropic / uniaxial-hyperbolic / "
                                   "gyrotropic), node counts log-uniform in [1024, 32768] (1D kx or 2D kρ x 8 φ), "
                                   "4 z rows x 4x4 lateral offsets each", "stacks": len(tr), "nodes_per_step": nodes,
                       "entries_per_step": int(entries), "precision": prec,
                       "calls": "ytf_plan_run + ytf_plan_wait: one CUDA graph per step (H2D of nodes and "
                                "coordinates, persistent node-solve kernels, batched synthesis, D2H of G)",
                       "tune": rec["tune"], "tune_class": autotune.config_class(items, syn),
                       "tuning_s": round(tune_s, 2), "tune_measured": rec.get("measured"),
                       "default_tune_ms": rec.get("default_ms"), "node_solve_passes": info["passes"]},
            "max_rel_err_vs_oracle": err, "max_rel_diff_vs_per_item_calls": err_calls,
            "e2e": {"value": entries / (wall_ms * 1e-3), "unit": "entries/s", "h2d_bytes_per_step": info["h2d_bytes"],
                    "d2h_bytes_per_step": info["d2h_bytes"], "ms_per_step": wall_ms},
            "per_item_calls_ms_per_step": calls_ms, "clocks": clk.summary(),
            "nodes_per_s": nodes / (ms * 1e-3),
            "kernels_per_step": {k: v[1] // max(args.steps, 1) for k, v in sorted(prof.items())},
            "gpu_launches": int(sum(v[1] for v in prof.values()))}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------------------
# The headline workload: learned-adaptive vs plain quadrature
# --------------------------------------------------------------------------------------
LEARNED_METRIC = "G(ρ,z,z') entries/s at ≤1e-6 rel err: learned-adaptive vs plain, 1 B200"
N_TEST, CHUNK = 4096, 256          # held-out stacks; stacks per step
N_RHO, N_ZOBS = 256, 64            # the observation grid of the 3-layer dipole problem
Z_SRC = 20.0                       # nm: vertical dipole above the film
ENTRIES_PER_STACK = N_RHO * N_ZOBS * 9
N_TRAIN_SAMPLES, N_SCAN = 10_000_000, 2048
N_CHECK = 512                      # stacks whose returned G is checked against a converged reference


def learned_stacks(n=N_TEST, seed=SEED + 5):
    """The held-out stacks: air / uniaxial film / substrate (the film's losses from sharp to
    broad guided modes, d 20-100 nm), λ U[450, 750] nm."""
    from yellowthinfilms_b200 import learned as L
    rng = np.random.default_rng(seed)
    return [L.film_stack(rng) for _ in range(n)]


def learned_obs(lam):
    """(z rows, radii, h_min): 64 heights uniform over 0-200 nm above the film, 256 radii
    log-spaced over 0.01-5 λ. h_min is the shortest path of a reflected wave, source height
    plus the lowest observer height (20 nm), so Kcut = 25 / h_min."""
    z = np.linspace(0.0, 200.0, N_ZOBS)
    rho = np.geomspace(0.01 * lam, 5.0 * lam, N_RHO)
    return z, rho, Z_SRC + float(z.min())


def learned_problem(st, lam, sto, precision="int8x3"):
    z, rho, h_min = learned_obs(lam)
    return dict(stack=sto, layers=st, k0=2 * np.pi / lam, source_layer=1, zsrc_local=Z_SRC, z=z, rho=rho,
                terms="scattered", h_min=h_min, rho_max=float(rho[-1]), precision=precision)


LEARNED_CONFIG = {"workload": f"learned adaptive quadrature vs the plain fixed rule: {N_TEST} held-out seeded air / "
                              f"uniaxial film / substrate stacks, vertical dipole {Z_SRC:g} nm above the film, "
                              f"{N_RHO} ρ log-spaced over 0.01-5 λ x {N_ZOBS} heights uniform over 0-200 nm x 9 "
                              f"components (scattered term); h_min = 20 nm (source height + lowest observer)",
                  "held_out_stacks": N_TEST, "stacks_per_step": CHUNK, "entries_per_stack": ENTRIES_PER_STACK,
                  "gzz_entries_per_stack": N_RHO * N_ZOBS, "train_samples": N_TRAIN_SAMPLES, "tolerance": 1e-6,
                  "seed": SEED,
                  "l2": "per-step working set (the caches and G of 256 stacks, several GB) larger than L2"}


def cpu_learned(stacks, threads=None):
    """The reference's own method on the CPU (the oracle): per stack the scanned point rule
    (kspace_features with the pole scan + fixed_kρ_rule at rtol 1e-6), the 1D cache and
    closed_form_G on the full observation grid. Returns (seconds per stack, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ytf_oracle as oracle
    oracle.set_threads(threads or os.cpu_count() or 1)
    ts = []
    for st, lam in stacks:
        k0 = 2 * np.pi / lam
        z, rho, h_min = learned_obs(lam)
        t = time.perf_counter()
        k, w, _ = oracle.fixed_grid_1d(st, k0, 1, h_min=h_min, rho_max=float(rho[-1]), scan=True, rtol=1e-6)
        c = oracle.build_cavity_transfer_1d(st, k0, 1, k, w, obs_layers=[1])
        oracle.closed_form_G(c, 1, Z_SRC, z, rho, [0.0], terms="scattered")
        ts.append(time.perf_counter() - t)
    return ts, oracle.num_threads()


def run_reference_learned(args):
    """The reference arm of the headline workload: one held-out stack per step through the
    CPU restatement of the reference's method (no product library in this process)."""
    if rank_env()[0] != 0:
        return 0
    stacks = learned_stacks(args.warmup + args.steps)
    cpu_learned(stacks[:args.warmup])
    ts, cores = cpu_learned(stacks[args.warmup:])
    t = float(np.sum(ts))
    value = args.steps * ENTRIES_PER_STACK / t
    line = {"metric": LEARNED_METRIC, "value": value, "unit": "entries/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded)", "impl": "reference",
            "config": dict(LEARNED_CONFIG, precision="fp64 (CPU oracle)"),
            "cpu_baseline": {"value": value, "unit": "entries/s", "cores": cores, "kind": "port",
                             "sample": f"one held-out stack per step ({ENTRIES_PER_STACK} entries): the reference's "
                                       "scanned fixed rule, the 1D cache and closed_form_G, timed whole"},
            "e2e": {"value": value, "unit": "entries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# FP64 operations per (ρ, k) pair of k_aimg_bessel3 (J_0, J_1 by Hankel's asymptotic pair from
# x = 25 and the CUDA math library below, J_2 by series or recurrence, digits): ncu's DFMA x 2 +
# DMUL + DADD of one grouped launch divided by its (ρ, k) slots, 3.32e9 / 23.05e6
AIMG_FP64_PER_PAIR = 144.0
# DRAM bytes per node synthesised of the grouped kernels (dram__bytes_read + write of one ncu
# capture of `--workload synth --stacks 8 --group-bytes 1073741824`, one group of 89,144 nodes;
# traffic grows with the nodes of a launch), scaled to a launch's nodes
TRAFFIC_PER_NODE = {"k_gemm_i8_img": 6316.0, "k_aimg_bessel3": 1748.0, "k_coef1d": 4581.0, "k_bimg_real": 10357.0}


def learned_roofline(name, prof, nodes_synth):
    """Roofline entry of one kernel of the learned step's synthesis from its CUDA-event time in
    the profiled step: the int8x3 contraction against the sustained bf16 tensor peak (its
    algorithmic flops: 2 x radii x 1152 real coefficient columns per node synthesised), the
    J_n image kernel against the nominal FP64 peak (its counted FP64 operations)."""
    roof = {"kernel": name, "bound": None, "achieved": None, "peak": None, "unit": None, "frac": None,
            "traffic": TRAFFIC.get(name)}
    if name not in prof or not prof[name][1]:
        return roof
    t_k, nl = prof[name][0] * 1e-3, prof[name][1]
    if name in TRAFFIC_PER_NODE:
        roof["traffic"] = TRAFFIC_PER_NODE[name] * nodes_synth / nl
        roof["traffic_note"] = "bytes per launch: ncu bytes per node (89,144-node capture) x nodes per launch"
    peaks = measured_peaks()
    if name in ("k_gemm_i8_img", "k_bessel_i8"):
        flops = 2.0 * N_RHO * (18 * N_ZOBS) * nodes_synth  # the 9 stored complex coefficient columns per height
        peak, src = peaks["bf16_sustained"]
        roof.update(bound="tensor", achieved=flops / t_k / 1e12, peak=peak, unit="TFLOP/s",
                    frac=flops / t_k / 1e12 / peak, peak_source=src, launches=nl,
                    work=f"2 x {N_RHO} radii x 1152 real coefficient columns x nodes synthesised "
                         f"({int(nodes_synth)} over the chunk's syntheses) = {flops:.3e} flop in {nl} launches")
    elif name == "k_aimg_bessel3":
        ops = AIMG_FP64_PER_PAIR * N_RHO * nodes_synth
        roof.update(bound="fp64", achieved=ops / t_k / 1e12, peak=FP64_NOMINAL, unit="TFLOP/s",
                    frac=ops / t_k / 1e12 / FP64_NOMINAL, peak_source="nominal FP64; no measured FP64 peak",
                    launches=nl, work=f"{AIMG_FP64_PER_PAIR:.0f} FP64 ops (ncu count) x {N_RHO} radii x "
                                      f"{int(nodes_synth)} nodes synthesised = {ops:.3e} in {nl} launches")
    return roof


def run_learned(args):
    """Learned adaptive quadrature vs the plain fixed rule. The node-placement MLP is trained
    on 1e7 solver samples (timed separately); then every step takes one chunk of 256 held-out
    stacks through both methods, each to a G accurate to 1e-6: the learned rule (network
    proposals, exact window sampling, fixed_kρ_rule, the check against G on the same panels
    at Gauss–Legendre order 10, plain halving on rejection) and the plain rule without pole
    knowledge halved until two levels agree. Every node of both is solved exactly; both synthesise with the int8x3 tensor-core contraction.
    `value` is the learned method's entries/s with G left in HBM, `e2e` the same with every G
    copied to page-locked host memory inside the timed region; `plain_entries_per_s` is the
    plain method on the same stacks. A seeded sample of >= 512 returned G of both methods is
    checked against a converged reference (scanned rule at rtol 1e-10, halved, FP64
    synthesis)."""
    import torch
    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    from yellowthinfilms_b200 import api
    from yellowthinfilms_b200 import learned as L
    ctx = api.Context(local)
    api._default_ctx = ctx
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    prec = args.precision if args.precision != "split_bf16" else "int8x3"

    # training (outside the timed region, reported beside it)
    n_train = args.train_samples // N_SCAN
    t = time.perf_counter()
    X, T = L.training_set(n_train, n_k=N_SCAN, seed=SEED, ctx=ctx)
    t_data = time.perf_counter() - t
    net = L.new_network(seed=SEED, device=local)
    net.set_stream(stream.cuda_stream)
    steps_train, batch = 2 * len(X) // 8192, 8192
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    del X, T
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    losses = net.train(Xd, Td, batch=batch, steps=steps_train, lr=1e-3, seed=SEED)
    b.record(stream)
    torch.cuda.synchronize()
    t_train = a.elapsed_time(b) * 1e-3
    del Xd, Td

    n_test = args.stacks
    stacks = learned_stacks(n_test)
    chunks = [list(range(c, min(c + CHUNK, n_test))) for c in range(0, n_test, CHUNK)]
    mine = chunks[rank::world] or chunks[:1]
    dev_stacks = {}

    # every step runs each method as --shares concurrent shares of the chunk (stacks dealt in turn), one
    # host thread, libytf context and CUDA stream each (learned.concurrent_shares), so that one
    # share's host steps overlap the other's device work; each share evaluates the network on its
    # own stacks with its own copy of the trained network (learned.copy_network)
    ns = max(1, args.shares)
    ctxs, streams, nets = [ctx], [stream], [net]
    for _ in range(ns - 1):
        c2, s2 = api.Context(local), torch.cuda.Stream()
        c2.set_stream(s2.cuda_stream)
        n2 = L.copy_network(net, device=local)
        n2.set_stream(s2.cuda_stream)
        ctxs.append(c2)
        streams.append(s2)
        nets.append(n2)

    def stack_of(i, c):
        if (i, c) not in dev_stacks:
            dev_stacks[(i, c)] = api.Stack(stacks[i][0], ctxs[c])
        return dev_stacks[(i, c)]

    def problems(idx, c=0):
        return [learned_problem(stacks[i][0], stacks[i][1], stack_of(i, c), prec) for i in idx]

    def interleave(parts):
        out = [None] * sum(len(q) for q in parts)
        for j, q in enumerate(parts):
            out[j::len(parts)] = q
        return out

    G_host = torch.empty((CHUNK, ENTRIES_PER_STACK), dtype=torch.complex128, pin_memory=True)
    per_step_check = min(CHUNK, -(-N_CHECK // max(args.steps, 1)))
    rng_check = np.random.default_rng(SEED + 11)
    kept = {}
    rec = dict(t_l=[], t_e2e=[], t_p=[], n_l=[], n_p=[], solved_l=[], solved_p=[], acc=0, h_l=[], h_p=[],
               entries=0, stacks=0, mutual=0.0)

    def step(s, timed):
        idx = mine[s % len(mine)]
        Ps = [problems(idx[j::ns], j) for j in range(ns)]
        P = interleave(Ps)
        sls, sps = [[0] * len(q) for q in Ps], [[0] * len(q) for q in Ps]
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            for s2 in streams[1:]:
                s2.wait_stream(stream)
            # each share evaluates the network on its own stacks with its own copy of it
            outs = L.concurrent_shares(
                lambda sh, c: L.learned_rules_batch(sh[2], sh[0], ctx=c, device=True, n_scan=N_SCAN, solved=sh[1]),
                [(Ps[j], sls[j], nets[j]) for j in range(ns)], ctxs, streams)
            for s2 in streams[1:]:
                stream.wait_stream(s2)
            ev[1].record(stream)
            outl = interleave(outs)
            for j, o in enumerate(outl):
                G_host[j].copy_(o[0].permute(4, 3, 2, 1, 0).reshape(-1), non_blocking=True)
            ev[2].record(stream)
            for s2 in streams[1:]:
                s2.wait_stream(stream)
            outs = L.concurrent_shares(lambda sh, c: L.plain_rules_batch(sh[0], ctx=c, device=True, solved=sh[1]),
                                       [(Ps[j], sps[j]) for j in range(ns)], ctxs, streams)
            for s2 in streams[1:]:
                stream.wait_stream(s2)
            ev[3].record(stream)
            outp = interleave(outs)
        torch.cuda.synchronize()
        sl, sp = interleave(sls), interleave(sps)
        if not timed:
            return
        rec["t_l"].append(ev[0].elapsed_time(ev[1]) * 1e-3)
        rec["t_e2e"].append(ev[0].elapsed_time(ev[2]) * 1e-3)
        rec["t_p"].append(ev[2].elapsed_time(ev[3]) * 1e-3)
        rec["entries"] += len(P) * ENTRIES_PER_STACK
        rec["stacks"] += len(P)
        rec["solved_l"] += sl
        rec["solved_p"] += sp
        for j, (ol, op) in enumerate(zip(outl, outp)):
            rec["n_l"].append(len(ol[1]))
            rec["n_p"].append(len(op[1]))
            rec["acc"] += int(ol[3])
            rec["h_l"].append(ol[4])
            rec["h_p"].append(op[3])
            rec["mutual"] = max(rec["mutual"], float(torch.linalg.vector_norm(ol[0] - op[0]) /
                                                     torch.linalg.vector_norm(op[0])))
        for j in rng_check.choice(len(P), min(per_step_check, len(P)), replace=False):
            i = idx[int(j)]
            if i not in kept:
                kept[i] = (outl[int(j)][0].clone(), outp[int(j)][0].clone())
        del outl, outp

    # the objects of the setup (held-out stacks, network, imported modules) leave the cyclic
    # collector's generations, so that a full collection during a step does not re-scan them
    gc.collect()
    gc.freeze()
    for s in range(args.warmup):
        step(s, False)
    with Clocks(local) as clk:
        for s in range(args.steps):
            step(args.warmup + s, True)
    gc.unfreeze()
    t_l, t_e2e, t_p = (max_over_ranks(float(np.sum(rec[k])), dist, f"cuda:{local}") for k in ("t_l", "t_e2e", "t_p"))
    entries = rec["entries"]
    value = job_rate(entries, world, t_l * 1e3)
    e2e = job_rate(entries, world, t_e2e * 1e3)
    plain = job_rate(entries, world, t_p * 1e3)

    # a profiled pass of one chunk of the learned method (untimed): per-kernel CUDA-event times
    sl = [0] * CHUNK
    ctx.profile(True)
    L.learned_rules_batch(net, problems(mine[0]), ctx=ctx, device=True, n_scan=N_SCAN, solved=sl)
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)

    # parity: the sampled returned G of both methods against a converged reference: the scanned
    # rule at rtol 1e-10, halved until two successive levels agree to 1e-10 (FP64 synthesis)
    err_l = err_p = 0.0
    worst = None
    ref_unconverged = 0
    checked = sorted(kept)
    if not args.no_check:
        for c0 in range(0, len(checked), 32):
            part = checked[c0:c0 + 32]
            P = [learned_problem(stacks[i][0], stacks[i][1], stack_of(i, 0), "fp64") for i in part]
            rules, panels = [], []
            for Pi in P:
                kr, wr, ir = api.point_kx_grid(Pi["stack"], Pi["k0"], 1, h_min=Pi["h_min"], rho_max=Pi["rho_max"],
                                               rtol=1e-10, ctx=ctx)
                rules.append((kr, wr))
                panels.append(ir["panels"])
            refs = [None] * len(P)
            L._refine_levels(P, range(len(P)), rules, panels, None, 1e-10, 3, 8, ctx, refs, True)
            for i, (gr, _, _, _, conv) in zip(part, refs):
                gl, gp = kept[i]
                nr = torch.linalg.vector_norm(gr)
                el, ep = float(torch.linalg.vector_norm(gl - gr) / nr), float(torch.linalg.vector_norm(gp - gr) / nr)
                ref_unconverged += int(not conv)
                if worst is None or max(el, ep) > worst[1]:
                    worst = (i, max(el, ep))
                err_l, err_p = max(err_l, el), max(err_p, ep)
            del refs
    cpu = None
    if rank == 0 and not args.no_check:
        ts, cores = cpu_learned(stacks[:2])
        cpu = {"value": 2 * ENTRIES_PER_STACK / float(np.sum(ts)), "unit": "entries/s", "cores": cores, "kind": "port",
               "sample": "2 held-out stacks, each whole: the reference's scanned fixed rule, the 1D cache and "
                         "closed_form_G (oracle, all host threads)"}

    # roofline of the dominant kernel of the profiled pass, and of the tensor-core contraction
    top = max(prof.items(), key=lambda kv: kv[1][0])[0] if prof else None
    nodes_synth = float(np.sum(sl))
    roof = learned_roofline(top, prof, nodes_synth)
    if top != "k_gemm_i8_img" and "k_gemm_i8_img" in prof:
        roof["contraction"] = learned_roofline("k_gemm_i8_img", prof, nodes_synth)
    nl, npl = np.asarray(rec["n_l"]), np.asarray(rec["n_p"])
    line = {"metric": LEARNED_METRIC, "value": value, "unit": "entries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_l / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": f"f64 node solve, {prec} tensor-core synthesis; MLP bf16 weights, fp32 accum",
            "data": "synthetic (seeded)", "impl": "learned-adaptive",
            "config": dict(LEARNED_CONFIG, precision=prec, shares_per_method=ns, steps_cover_stacks=rec["stacks"] * world,
                           held_out_stacks=n_test, train_samples=n_train * N_SCAN),
            "plain_entries_per_s": plain, "learned_vs_plain": t_p / t_l,
            "step_ms": {"learned": [round(1e3 * x, 2) for x in rec["t_l"]],
                        "plain": [round(1e3 * x, 2) for x in rec["t_p"]]},
            "gzz_entries_per_s": value / 9,
            "max_rel_err_vs_reference": max(err_l, err_p), "max_rel_err_learned": err_l, "max_rel_err_plain": err_p,
            "reference_checked_stacks": len(checked) * world, "max_rel_diff_learned_vs_plain": rec["mutual"],
            "reference": "scanned rule at rtol 1e-10, halved until two levels agree to 1e-10, FP64 synthesis",
            "reference_unconverged": ref_unconverged, "worst_checked_stack": worst[0] if worst else None,
            "nodes": {"mean_returned_learned": float(nl.mean()), "mean_returned_plain": float(npl.mean()),
                      "mean_solved_learned": float(np.mean(rec["solved_l"])),
                      "mean_solved_plain": float(np.mean(rec["solved_p"])),
                      "learned_proposals_accepted": rec["acc"], "stacks": rec["stacks"],
                      "mean_halvings_learned": float(np.mean(rec["h_l"])),
                      "mean_halvings_plain": float(np.mean(rec["h_p"]))},
            # host -> device per step: the rules' panel edges (16 B per 8-node panel; the nodes are
            # expanded on the device) and every stack's observation coordinates
            "e2e": {"value": e2e, "unit": "entries/s",
                    "h2d_bytes_per_step": int((2 * np.sum(rec["solved_l"]) + 8 * (N_RHO + N_ZOBS + 1) * rec["stacks"])
                                              / max(args.steps, 1)),
                    "d2h_bytes_per_step": CHUNK * ENTRIES_PER_STACK * 16,
                    "ms_per_step": 1e3 * t_e2e / max(args.steps, 1)},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary(),
            "gpu_launches": int(sum(v[1] for v in prof.values())) * args.steps,
            "gpu_launches_note": "launches of one profiled learned step (one chunk) x steps",
            "profiled_step_kernels_ms": {k: round(v[0], 3) for k, v in sorted(prof.items())},
            "training": {"samples": n_train * N_SCAN, "data_s": t_data, "train_s": t_train, "adam_steps": steps_train,
                         "batch": batch, "first_loss": float(losses[0]), "last_loss": float(np.mean(losses[-50:]))}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_bessel(args):
    """The Bessel synthesis at scale (one GPU): a film stack's 1D cache of 65536 nodes, G on
    4096 radii log-spaced over 0.001-10 λ x 256 observer heights (9,437,184 entries), timed
    for the contraction precision given and for FP64 beside it."""
    import torch
    from yellowthinfilms_b200 import api
    from yellowthinfilms_b200.materials import FlatOpticalLayer, IsotropicMaterial, UniaxialMaterial
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    lam = 600.0
    k0 = 2 * np.pi / lam
    st = [FlatOpticalLayer(IsotropicMaterial(1.0), 200.0),
          FlatOpticalLayer(UniaxialMaterial(-3.0 + 0.4j, 4.0 + 0.2j), 50.0),
          FlatOpticalLayer(IsotropicMaterial(2.25), 100.0)]
    stack = api.Stack(st, ctx)
    npan = 65536 // ORDER
    kx, wt = api.gl_rule([(20 * k0 * i / npan, 20 * k0 * (i + 1) / npan) for i in range(npan)], ORDER, ctx=ctx)
    cache = api.build_cavity_transfer_1d(stack, k0, 1, kx, wt, obs_layers=[1])
    rho = np.geomspace(0.001 * lam, 10 * lam, 4096)
    zo = np.linspace(0.5, 199.5, 256)
    prec = args.precision if args.precision != "split_bf16" else "int8x3"
    out = torch.empty(4096 * 256 * 9, dtype=torch.complex128, device="cuda")

    def run(p):
        for _ in range(args.warmup):
            api.closed_form_G(cache, 1, 20.0, zo, rho, [0.0], terms="scattered", precision=p, out=out)
        torch.cuda.synchronize()
        ctx.profile(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(0) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                api.closed_form_G(cache, 1, 20.0, zo, rho, [0.0], terms="scattered", precision=p, out=out)
            e1.record(stream)
            torch.cuda.synchronize()
        prof = ctx.profile_read()
        ctx.profile(False)
        return e0.elapsed_time(e1) / args.steps, prof, clk.summary(), out.cpu().numpy()

    ms, prof, clocks, G = run(prec)
    ms64, prof64, _, G64 = run("fp64")
    entries = G.size
    flops = 2.0 * 4096 * 65536 * 18 * 256  # the 9 stored complex coefficient columns (18 real) per height
    name = "k_bessel_i8" if prec == "int8x3" else "k_dgemm_nt"
    t_k = prof[name][0] / prof[name][1] * 1e-3 if name in prof else None
    peak, src = measured_peaks()["bf16_sustained"]
    roof = {"kernel": name, "bound": "tensor" if prec == "int8x3" else "fp64",
            "achieved": flops / 3 / t_k / 1e12 if t_k else None, "unit": "TFLOP/s",
            "peak": peak if prec == "int8x3" else FP64_NOMINAL, "traffic": None,
            "work": "2 x 4096 radii x 65536 nodes x 18 real columns x 256 heights = 2.47e12 flop over the 3 orders "
                    "(one launch per order: a third each)",
            "peak_source": src if prec == "int8x3" else "nominal FP64"}
    if roof["achieved"]:
        roof["frac"] = roof["achieved"] / roof["peak"]
        if prec == "int8x3":
            roof["executed_frac_of_int8_peak"] = 6 * roof["achieved"] / (2 * peak)
    line = {"metric": METRIC, "value": entries / (ms * 1e-3), "unit": "entries/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE[prec], "data": "synthetic (seeded)",
            "config": {"workload": "Bessel synthesis: film stack, 65536 nodes, 4096 radii (0.001-10 λ) x 256 heights "
                                   "x 9 components, scattered term", "entries_per_step": int(entries),
                       "precision": prec},
            "fp64_entries_per_s": entries / (ms64 * 1e-3), "speedup_vs_fp64": ms64 / ms,
            "max_rel_err_vs_fp64": float(np.linalg.norm(G - G64) / np.linalg.norm(G64)),
            "roofline": roof, "clocks": clocks,
            "kernels_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in sorted(prof.items())},
            "fp64_kernels_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in sorted(prof64.items())}}
    print(json.dumps(line), flush=True)
    return 0


def run_synth(args):
    """The grouped 1D int8x3 synthesis alone (ytf_green_batch): --stacks held-out stacks of the
    learned workload (default 64) with their plain fixed rules (point_kx_grid without the
    scan), G on the dipole problem's 256 radii x 64 heights (scattered term, device outputs),
    all items in one batched call per step; --group-bytes bounds a group's workspace. Reports
    entries/s, ns per node and the per-kernel CUDA-event split of a profiled step, and the
    largest relative difference to the FP64 synthesis of the same items."""
    import torch
    from yellowthinfilms_b200 import api
    from yellowthinfilms_b200 import learned as L
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    api._default_ctx = ctx
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    if args.group_bytes:
        ctx.set_group_bytes(args.group_bytes)
    n = args.stacks if args.stacks != N_TEST else 64
    P = [learned_problem(st, lam, api.Stack(st, ctx), "int8x3") for st, lam in learned_stacks(n)]
    panels = api.rule_panels_batch([dict(stack=q["stack"], omega=q["k0"], source_layer=1, h_min=q["h_min"],
                                         rho_max=q["rho_max"]) for q in P], ctx=ctx)
    rules = api.gl_rule_batch([(pn, L._sing(q)) for pn, q in zip(panels, P)], ORDER, ctx=ctx, device=True)
    caches = api.build_cavity_transfer_batch([dict(stack=q["stack"], omega=q["k0"], source_layer=1, kx_nodes=k,
                                                   wt_nodes=w, obs_layers=[1]) for q, (k, w) in zip(P, rules)], ctx=ctx)
    nodes = int(sum(len(k) for k, _ in rules))
    outs = [torch.empty(N_RHO * N_ZOBS * 9, dtype=torch.complex128, device="cuda") for _ in P]
    items = [dict(cache=c, obs_layer=1, zsrc_local=q["zsrc_local"], z_obs=q["z"], xs=q["rho"], ys=[0.0],
                  terms="scattered", precision="int8x3", out=o) for c, q, o in zip(caches, P, outs)]
    for _ in range(args.warmup):
        api.closed_form_G_batch(items)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            api.closed_form_G_batch(items)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    ctx.profile(True)
    api.closed_form_G_batch(items)
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    G8 = [o.clone() for o in outs]
    api.closed_form_G_batch([dict(it, precision="fp64") for it in items])
    err = max(float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)) for a, b in zip(G8, outs))
    entries = len(P) * ENTRIES_PER_STACK
    roof = learned_roofline("k_gemm_i8_img", prof, nodes)
    line = {"metric": METRIC, "value": entries / (ms * 1e-3), "unit": "entries/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE["int8x3"], "data": "synthetic (seeded)",
            "config": {"workload": f"grouped 1D int8x3 synthesis: {len(P)} held-out film stacks of the learned workload "
                                   f"on their plain fixed rules ({nodes} nodes), {N_RHO} radii x {N_ZOBS} heights x 9 "
                                   "components each, one batched call per step",
                       "items": len(P), "nodes": nodes, "group_bytes": args.group_bytes or "default (4 GiB)"},
            "ns_per_node": ms * 1e6 / nodes, "max_rel_err_vs_fp64": err, "roofline": roof, "clocks": clk.summary(),
            "kernels_ms_per_step": {k: round(v[0], 4) for k, v in sorted(prof.items())},
            "kernels_note": "per-kernel CUDA-event times of one separately profiled step"}
    print(json.dumps(line), flush=True)
    return 0


def run_contour(args):
    """The config-1 path: vertical dipole 20 nm above the uniaxial film, 4096 nodes on the
    deformed contour (512 GL-8 panels, indentation 0.05 k0) to 20 k0, G at 256 radii
    (6-3000 nm, log) x 64 heights (0-200 nm); one step = transfer build + closed_form_G."""
    import torch
    from yellowthinfilms_b200 import api
    from yellowthinfilms_b200.materials import FlatOpticalLayer, IsotropicMaterial, UniaxialMaterial
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    lam = 600.0
    k0 = 2 * np.pi / lam
    layers = [FlatOpticalLayer(IsotropicMaterial(1.0), 200.0),
              FlatOpticalLayer(UniaxialMaterial(-3.0 + 0.4j, 4.0 + 0.2j), 50.0),
              FlatOpticalLayer(IsotropicMaterial(2.25), 100.0)]
    st = api.Stack(layers, ctx)
    k, w = api.contour_rule(k0, npanels=512, order=8)
    rho = np.geomspace(6.0, 3000.0, 256)
    zo = np.linspace(0.0, 200.0, 64)
    out = torch.empty(256 * 64 * 9, dtype=torch.complex128, device="cuda")

    prec = "int8x3" if args.precision != "fp64" else "fp64"

    def step(p):
        c = api.build_cavity_transfer_1d_contour(st, k0, 1, k, w, obs_layers=[1])
        api.closed_form_G(c, 1, 20.0, zo, rho, [0.0], out=out, precision=p)

    def run(p):
        for _ in range(args.warmup):
            step(p)
        torch.cuda.synchronize()
        ctx.profile(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(0) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                step(p)
            e1.record(stream)
            torch.cuda.synchronize()
        prof = ctx.profile_read()
        ctx.profile(False)
        return e0.elapsed_time(e1) / args.steps, prof, clk.summary(), out.clone()

    ms64, prof64, clocks64, G64 = run("fp64")
    ms, prof, clocks, G = run(prec) if prec != "fp64" else (ms64, prof64, clocks64, G64)
    line = {"metric": METRIC, "value": 256 * 64 * 9 / (ms * 1e-3), "unit": "entries/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "c128 node solve; complex J_n; " + ("int8x3 tensor-core contraction (Re J, Im J digit images)"
                                                         if prec != "fp64" else "FP64 contraction"),
            "fp64_entries_per_s": 256 * 64 * 9 / (ms64 * 1e-3),
            "max_rel_diff_vs_fp64": float(torch.linalg.vector_norm(G - G64) / torch.linalg.vector_norm(G64)),
            "fp64_kernels_ms_per_step": {kk: round(v[0] / args.steps, 4) for kk, v in sorted(prof64.items())},
            "data": "synthetic (the config-1 stack)",
            "config": {"workload": "vertical dipole 20 nm above a uniaxial film (εo = -3+0.4i, εe = 4+0.2i, 50 nm) on "
                                   "glass, λ = 600 nm; 4096 nodes on kρ = t - 0.05 i k0 sin(π t / 20 k0); 256 ρ x 64 z",
                       "entries_per_step": 256 * 64 * 9, "gzz_entries_per_step": 256 * 64},
            "gzz_entries_per_s": 256 * 64 / (ms * 1e-3), "clocks": clocks,
            "kernels_ms_per_step": {kk: round(v[0] / args.steps, 4) for kk, v in sorted(prof.items())}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--shares", type=int, default=2,
                    help="learned workload: concurrent shares of a chunk per method (host thread, context, stream each)")
    ap.add_argument("--group-bytes", type=int, default=0,
                    help="synth workload: workspace bound of one synthesis group (0: the library default)")
    ap.add_argument("--workload", default="learned", choices=["learned", "gyro32", "uneven", "bessel", "contour",
                                                              "synth"],
                    help="learned: learned adaptive quadrature vs the plain fixed rule on 4096 held-out stacks "
                         "(default, the headline metric); gyro32: the 8-layer stack at 32 wavelengths; uneven: 1024 "
                         "uneven stacks; bessel: the 1D Bessel synthesis at 4096 radii x 65536 nodes x 256 heights; "
                         "contour: the config-1 path on the deformed contour")
    ap.add_argument("--stacks", type=int, default=N_TEST,
                    help="learned workload: held-out stacks (default 4096; fewer only for profiling runs)")
    ap.add_argument("--train-samples", type=int, default=N_TRAIN_SAMPLES,
                    help="learned workload: training samples (default 1e7; fewer only for profiling runs)")
    ap.add_argument("--retune", action="store_true",
                    help="uneven workload: tune the plan again even if the tuning database has its class")
    ap.add_argument("--calls", default="plan", choices=["plan", "batched", "per-call"],
                    help="plan: the whole step as one CUDA graph (ytf_plan_*, default); batched: one "
                         "ytf_transfer_batch + one ytf_green_batch call per step; per-call: one build + "
                         "synthesis call per wavelength")
    ap.add_argument("--per-call", action="store_true", help="the same as --calls per-call")
    ap.add_argument("--precision", default="int8x3", choices=list(DTYPE),
                    help="lateral contraction: int8 tensor cores (three base-256 digits, exact INT32 "
                         "accumulation), split-BF16 tensor cores (FP32 accumulation) or FP64 CUDA cores")
    args = ap.parse_args()
    if args.per_call:
        args.calls = "per-call"
    if args.impl == "reference":
        if args.workload == "learned":
            return run_reference_learned(args)
        if args.workload == "gyro32":
            return run_reference(args)
        print(json.dumps({"impl": "reference", "unavailable": f"no reference arm for the {args.workload} workload; "
                                                              "the reference arms are learned and gyro32"}))
        return 0
    if args.workload == "uneven":
        return run_uneven(args)
    if args.workload == "learned":
        return run_learned(args)
    if args.workload == "synth":
        return run_synth(args)
    if args.workload == "bessel":
        return run_bessel(args)
    if args.workload == "contour":
        return run_contour(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
