"""Autotuner for the sweep solver: frequencies per batch, LU outer panel width
and the tensor-core tile widths of the LU's trailing updates.

For a given geometry it times short sweeps over the candidate settings and
keeps the fastest whose refinement still converges (no FP64 fallback): first
(batch, panel width) with 256-column tiles, then the tile-width pairs
(128 or 256 complex columns per CTA pair, for the panel chain's K = 64
updates and for the outer panels' updates) and resident variants at the
winning batch and panel width, then the batches per shared factorization.  The winners are cached in ``tuned.json`` next to this file, keyed by
the Ne bucket (powers of two) and the GPU's SM count; ``tuned_opts()`` looks
them up so that a SweepPlan created without explicit options uses them.

    python -m autotune  (from the package directory) or tune(plan_args, freqs)
"""
from __future__ import annotations

import json
import math
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuned.json")
BATCHES = (0, 16, 32)    # 0: the library's automatic, balanced batches
PANELS = (128, 256, 512)
# (tile_chain, tile_bulk, resident_chain, resident_bulk)
TILES = ((256, 256, 0, 0), (128, 256, 0, 0), (256, 128, 0, 0), (128, 128, 0, 0), (256, 256, 1, 0),
         (256, 256, 0, 1), (256, 256, 1, 1))
# batches per shared factorization (0: the library's automatic choice)
SHARES = (0, 2, 4, 6, 8)


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
    """(batch, lu_nb, tile_chain, tile_bulk, resident_chain, resident_bulk,
    share_factors) for this size on this GPU, or None when untuned (0 = the
    library's default)."""
    try:
        sms = sms or _sms()
    except Exception:  # noqa: BLE001 - no torch/GPU: no table lookup
        return None
    e = load_table().get(_key(Ne, sms))
    return ((e["batch"], e["lu_nb"], e.get("tile_chain", 0), e.get("tile_bulk", 0), e.get("resident_chain", 0),
             e.get("resident_bulk", 0), e.get("share_factors", 0)) if e else None)


def _time(plan_args, freqs, repeats, **kw):
    from .api import SweepPlan, sweep_opts
    from . import _native
    try:
        plan = SweepPlan(*plan_args, opts=sweep_opts(nfreq_hint=len(freqs), **kw))
    except _native.MexError as e:
        if e.identifier != "efie:nomem":
            raise
        return len(plan_args[2]), None   # a batch too large for this GPU: no candidate
    plan.run(freqs)                                  # warm-up: workspaces, kernels, graph
    t0 = time.perf_counter()
    ok = True
    for _ in range(repeats):
        plan.run(freqs)
        ok = ok and plan.stats["n_fp64_fallback"] == 0
    dt = time.perf_counter() - t0
    Ne = plan.Ne
    plan.close()
    return Ne, ((repeats * len(freqs) / dt) if ok else None)


def tune(plan_args, freqs, candidates=None, repeats=1, save=True, tiles=True, shares=True):
    """Time every (batch, lu_nb) candidate on the sweep of ``freqs``, then
    (with ``tiles``) the tile-width pairs and resident variants at the
    winner, then (with ``shares``) the batches per shared factorization.

    plan_args: the positional arguments of SweepPlan (geometry .. Z0).
    Returns (best, results): best = (batch, lu_nb, tile_chain, tile_bulk,
    resident_chain, resident_bulk, share_factors), results[best-like tuple]
    = points/s or None.  A later stage's variant replaces the earlier
    winner only if it is more than 1 % faster (the run-to-run noise of a
    sweep).
    """
    cands = candidates or [(b, p) for b in BATCHES for p in PANELS]
    results = {}
    Ne = None

    def run(key):
        nonlocal Ne
        if key not in results:
            b, p, tc, tb, rc, rb, g = key
            Ne, results[key] = _time(plan_args, freqs, repeats, batch=b, lu_nb=p, tile_chain=tc, tile_bulk=tb,
                                     resident_chain=rc, resident_bulk=rb, share_factors=g)

    def pick(keys, base):
        good = {k: results[k] for k in keys if results.get(k)}
        if not good:
            return None
        best = max(good, key=good.get)
        if results.get(base) and good[best] < 1.01 * results[base]:
            return base
        return best

    for batch, panel in cands:
        run((batch, panel, 256, 256, 0, 0, 0))
    good = {k: v for k, v in results.items() if v}
    best = max(good, key=good.get) if good else None
    if best and tiles:
        keys = [best[:2] + t + (0,) for t in TILES]
        for k in keys:
            run(k)
        best = pick(keys, best[:2] + (256, 256, 0, 0, 0))
    if best and shares:
        keys = [best[:6] + (g,) for g in SHARES]
        for k in keys:
            run(k)
        best = pick(keys, best[:6] + (0,))
    if save and best:
        table = load_table()
        table[_key(Ne, _sms())] = dict(batch=best[0], lu_nb=best[1], tile_chain=best[2], tile_bulk=best[3],
                                       resident_chain=best[4], resident_bulk=best[5], share_factors=best[6],
                                       points_per_s=results[best],
                                       candidates={"/".join(str(x) for x in k): v for k, v in results.items()})
        with open(TABLE, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
    return best, results


def _patch_problem(Npx, Npy, Ngx, Ngy, Lp=30e-3, Wp=38e-3, Lg=60e-3, Wg=60e-3, h=1.6e-3):
    """SweepPlan arguments of a two-plate patch (reference GPU option set,
    main_patch_gpu_mex_sweep_l.m:50-56) through the package's producers."""
    from .api import build_rwg_interior, efie_precompute_pack, make_patch_with_ground_mesh, \
        pick_port_edge_by_point_and_layer
    import numpy as np
    V, F, _, _ = make_patch_with_ground_mesh(Lp, Wp, Lg, Wg, h, Npx, Npy, Ngx, Ngy, vertex_order="grid")
    r = build_rwg_interior({"V": V, "F": F})
    pe = pick_port_edge_by_point_and_layer(r, (0.0, -7e-3, +h / 2), +1)
    ge = pick_port_edge_by_point_and_layer(r, (0.0, -7e-3, -h / 2), -1)
    pre = efie_precompute_pack({"V": V, "F": F}, dict(quad_order=2, near_sing_eps=1.2, self_subdiv=2,
                                                      self_alpha=0.20, near_subdiv=1, near_alpha=0.15,
                                                      near_order=2))
    mu0 = 4e-7 * math.pi
    eps0 = 1.0 / (mu0 * 299792458.0 ** 2)
    return [V, F, r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
            r["Ap"], r["Am"], r["len"], pre, mu0, eps0, pe, ge, 1.0, 1.5 * float(np.mean(r["len"])), 50.0]


if __name__ == "__main__":
    # python -m <package>.autotune [grid ...]: tune the 101-point 2-3 GHz sweep
    # of the patch 38x30 mm over a 60x60 mm ground for each grid (default:
    # the 32x24 / 40x40 mesh, Ne 6968)
    import sys
    import numpy as np
    grids = [tuple(int(x) for x in a.split("x")) for a in sys.argv[1:]] or [(32, 24, 40, 40)]
    for g in grids:
        best, res = tune(_patch_problem(*g), np.linspace(2e9, 3e9, 101))
        print(json.dumps({"grid": g, "best": best, "results": {"/".join(str(x) for x in k): v for k, v in res.items()}}))
