"""Autotuner of uneven-batch plans (BatchPlan / ytf_plan_*). No counterpart in the
reference, which runs one build and one synthesis per item on the host's threads.

The tunables are the fields of ytf_tune: threads per CTA of the persistent node-solve
kernels (``block``), their grid in CTAs per SM (``ctas_per_sm``), units per node-solve tile
(``tile``), nodes per synthesis work unit (``chunk``) and the synthesis grid
(``synth_ctas_per_sm``). The tuner measures the device time of the plan's graph
(``BatchPlan.retune`` + ``run``/``wait``, CUDA events) for candidates in a coordinate
descent from the defaults: one parameter at a time over its candidate values, keeping the
best, in the order of ``ORDER``. The choice is persisted in a JSON file keyed by
(architecture, configuration class), so a later plan of the same class on the same kind of
GPU starts from it without measuring.

The configuration class buckets the batch by what sets the best tiles: the item count and
the mean nodes per item (powers of two), the largest layer count (up to 8, 16 or 32), the
share of 2D items (none, some, all) and the largest pixel set.
"""
from __future__ import annotations

import json
import math
import os
from typing import Callable, Optional

DEFAULT = dict(block=128, ctas_per_sm=4, tile=1024, chunk=2048, synth_ctas_per_sm=2)
CANDIDATES = dict(ctas_per_sm=(1, 2, 4, 8), block=(128, 256), tile=(256, 1024, 4096), chunk=(512, 2048, 8192),
                  synth_ctas_per_sm=(1, 2, 4))
ORDER = ("ctas_per_sm", "block", "tile", "chunk", "synth_ctas_per_sm")


def cache_path() -> str:
    """The tuning database: $YTF_TUNE_CACHE, else ~/.cache/yellowthinfilms_b200/tune.json."""
    p = os.environ.get("YTF_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "yellowthinfilms_b200", "tune.json")


def load(path: Optional[str] = None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as f:
            db = json.load(f)
        return db if isinstance(db, dict) else {}
    except (OSError, ValueError):
        return {}


def save(db: dict, path: Optional[str] = None) -> None:
    path = path or cache_path()
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _log2_bucket(x: float) -> int:
    return int(math.floor(math.log2(x))) if x >= 1 else 0


def config_class(transfer_items, green_items) -> str:
    """Bucket string of a batch (see the module docstring)."""
    nb = len(transfer_items)
    nodes, layers, n2d, pix = 0, 0, 0, 0
    for it, g in zip(transfer_items, green_items):
        if "kr_nodes" in it:
            nodes += len(it["kr_nodes"]) * len(it["phi_nodes"])
            n2d += 1
        else:
            nodes += len(it["kx_nodes"])
        st = it["stack"]
        nl = len(st.layers) if hasattr(st, "layers") else len(st)
        layers = max(layers, nl)
        if not isinstance(g, dict):
            g = dict(zip(("obs_layer", "zsrc_local", "z_obs", "xs", "ys"), g))
        pix = max(pix, len(g["xs"]) * len(g["ys"]))
    mean = nodes / max(nb, 1)
    lb = 8 if layers <= 8 else (16 if layers <= 16 else 32)
    share = "none" if n2d == 0 else ("all" if n2d == nb else "some")
    return f"items{_log2_bucket(nb)}_nodes{_log2_bucket(mean)}_layers{lb}_2d-{share}_pix{_log2_bucket(pix)}"


def device_arch(device: int = 0) -> str:
    """sm_XY and the device name (torch's view of the device)."""
    import torch
    p = torch.cuda.get_device_properties(device)
    return f"sm_{p.major}{p.minor} {p.name}"


def descend(measure: Callable[[dict], float], start: Optional[dict] = None, candidates=CANDIDATES,
            order=ORDER) -> tuple:
    """Coordinate descent: returns (best tune, its time, every (tune, time) measured)."""
    best = dict(DEFAULT)
    best.update(start or {})
    seen = {}

    def key(t):
        return tuple(sorted(t.items()))

    def m(t):
        k = key(t)
        if k not in seen:
            seen[k] = float(measure(dict(t)))
        return seen[k]

    best_ms = m(best)
    for name in order:
        for v in candidates[name]:
            t = dict(best)
            t[name] = v
            ms = m(t)
            if ms < best_ms:
                best, best_ms = t, ms
    return best, best_ms, [(dict(k), v) for k, v in seen.items()]


def measure_plan(plan, reps: int = 2) -> Callable[[dict], float]:
    """Device time (ms, the minimum of `reps` runs after one warm run) of the plan's graph
    under a tune."""
    def f(t):
        plan.retune(t)
        plan.run()
        plan.wait()
        best = float("inf")
        for _ in range(reps):
            plan.run()
            best = min(best, plan.wait())
        return best
    return f


def tuned_plan(transfer_items, green_items, ctx=None, arch: Optional[str] = None, path: Optional[str] = None,
               force: bool = False, reps: int = 2):
    """A BatchPlan with the persisted tiles of its (architecture, class), tuning and
    persisting them first when the class is new (or ``force``). Returns (plan, record)."""
    from .api import BatchPlan
    cls = config_class(transfer_items, green_items)
    arch = arch or device_arch(ctx.device if ctx is not None and hasattr(ctx, "device") else 0)
    k = f"{arch}|{cls}"
    db = load(path)
    rec = db.get(k)
    if rec is not None and not force:
        return BatchPlan(transfer_items, green_items, tune=rec["tune"], ctx=ctx), rec
    plan = BatchPlan(transfer_items, green_items, tune=None, ctx=ctx)
    best, ms, tried = descend(measure_plan(plan, reps))
    plan.retune(best)
    rec = dict(tune=best, ms=ms, measured=len(tried), default_ms=dict((tuple(sorted(t.items())), v) for t, v in tried)
               .get(tuple(sorted(DEFAULT.items()))))
    db[k] = rec
    save(db, path)
    return plan, rec
