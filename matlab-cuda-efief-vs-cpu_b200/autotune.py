"""Autotuner for the sweep solver: frequencies per batch and LU outer panel width.

For a given geometry it times short sweeps over the candidate settings and
keeps the fastest whose refinement still converges (no FP64 fallback).  The
winners are cached in ``tuned.json`` next to this file, keyed by the Ne bucket
(powers of two) and the GPU's SM count; ``tuned_opts()`` looks them up so
that a SweepPlan created without explicit options uses them.

    python -m autotune  (from the package directory) or tune(plan_args, freqs)
"""
from __future__ import annotations

import json
import math
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuned.json")
BATCHES = (8, 16, 32)
PANELS = (128, 256, 512)


def _key(Ne, sms):
    return "ne%d_sm%d" % (1 << max(0, math.ceil(math.log2(max(Ne, 1)))), sms)


def _sms():
    import torch
    return torch.cuda.get_device_properties(0).multi_processor_count


def load_table():
    try:
        with open(TABLE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def tuned_opts(Ne, sms=None):
    """(batch, lu_nb) for this size on this GPU, or None when untuned."""
    try:
        sms = sms or _sms()
    except Exception:  # noqa: BLE001 - no torch/GPU: no table lookup
        return None
    e = load_table().get(_key(Ne, sms))
    return (e["batch"], e["lu_nb"]) if e else None


def tune(plan_args, freqs, candidates=None, repeats=1, save=True):
    """Time every (batch, lu_nb) candidate on the sweep of ``freqs``.

    plan_args: the positional arguments of SweepPlan (geometry .. Z0).
    Returns (best, results) with results[(batch, lu_nb)] = points/s or None.
    """
    from .api import SweepPlan, sweep_opts
    cands = candidates or [(b, p) for b in BATCHES for p in PANELS]
    results = {}
    Ne = None
    for batch, panel in cands:
        plan = SweepPlan(*plan_args, opts=sweep_opts(batch=batch, lu_nb=panel))
        Ne = plan.Ne
        plan.run(freqs[:batch])                      # warm-up: workspaces, kernels
        t0 = time.perf_counter()
        ok = True
        for _ in range(repeats):
            plan.run(freqs)
            ok = ok and plan.stats["n_fp64_fallback"] == 0
        dt = time.perf_counter() - t0
        plan.close()
        results[(batch, panel)] = (repeats * len(freqs) / dt) if ok else None
    good = {k: v for k, v in results.items() if v}
    best = max(good, key=good.get) if good else None
    if save and best:
        table = load_table()
        table[_key(Ne, _sms())] = dict(batch=best[0], lu_nb=best[1], points_per_s=good[best],
                                       candidates={"%d/%d" % k: v for k, v in results.items()})
        with open(TABLE, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
    return best, results
