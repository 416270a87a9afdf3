#!/usr/bin/env python
"""Frequency-sweep throughput of the EFIE hot path on B200.

One step = one pass of the hot path (assemble Z, solve Z I = V, Zin/S11) over
a batch of frequency points of the workload; value = frequency points solved
per second over all ranks.  Multi-GPU runs are independent replicas (each
rank sweeps its own frequency points; no collective on the data path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cfg2] [--batch B] [--solver mixed|fp64]

The reference arm (--impl reference) times the reference's CPU path --
CPU_FAST assembly + backslash + Zin, restated in the oracle (C, OpenMP, all
host cores) with LAPACK from numpy -- on the same workload, one frequency
point per step; it also times the reference's own CUDA sweep (compiled from
its sources, oracle/_ref) on a bounded sample as ``ref_gpu``.
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = "matlab-cuda-efief-vs-cpu_b200"
METRIC = "freq points/s (assemble+LU+solve) mixed vs FP64 on B200 at rel Zin err ≤1e-6"

MU0 = 4.0 * math.pi * 1e-7
C0 = 299792458.0
EPS0 = 1.0 / (MU0 * C0 * C0)

# Workloads (synthetic geometry with the documented shapes; free space).
WORKLOADS = {
    # patch 38x30 mm on a 32x24 grid, 1.6 mm above a 60x60 mm ground on a 40x40 grid
    "cfg2": dict(Lp=30e-3, Wp=38e-3, Lg=60e-3, Wg=60e-3, h=1.6e-3, Np=(32, 24), Ng=(40, 40),
                 freqs=(2.0e9, 3.0e9, 101)),
    # same plates, patch 12x10 grid, ground 16x16 grid
    "cfg1": dict(Lp=30e-3, Wp=38e-3, Lg=60e-3, Wg=60e-3, h=1.6e-3, Np=(12, 10), Ng=(16, 16),
                 freqs=(2.0e9, 3.0e9, 11)),
    # large single design: patch 40x32 mm at 0.5 mm (80x64 grid) over a 90x90 mm ground as a
    # 40x40 grid (2.25 mm), h 1.6 mm: Ne = 19936
    "cfg5": dict(Lp=32e-3, Wp=40e-3, Lg=90e-3, Wg=90e-3, h=1.6e-3, Np=(80, 64), Ng=(40, 40),
                 freqs=(2.0e9, 3.0e9, 51)),
}
# Design-family workloads (surrogate.sample_designs): cfg3 sweeps 64 designs of
# uneven size (patch pitch 1.5 mm, ground pitch 3 mm: Ne 1390..3697) at 41
# points over f0 (1 +- 0.2); cfg4 trains the surrogate on solver samples of
# that distribution and runs adaptive sweeps against dense 201-point sweeps.
FAMILY = dict(n=64, seed=20261203, pitch=1.5e-3, ground_pitch=3e-3, nfreq=41)
RULE = {"ref": 0, "extract": -7}
SCHEME_NAME = {"ref": "reference cached subdivision + softening (GPU option set)",
               "extract": "Dunavant 7-point rule + analytic 1/R extraction on self/vertex-adjacent pairs"}
# The reference's GPU option set (main_patch_gpu_mex_sweep_l.m:50-56).
OPTS_REF_GPU = dict(quad_order=2, near_sing_eps=1.2, self_subdiv=2, self_alpha=0.20, near_subdiv=1,
                    near_alpha=0.15, near_order=2)


def _pkg():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    return importlib.import_module(PKG)


def build_inputs(m, wl):
    """Mesh, RWG, ports, prepack and sweep arguments through the product's producers."""
    w = WORKLOADS[wl]
    V, F, _, _ = m.make_patch_with_ground_mesh(w["Lp"], w["Wp"], w["Lg"], w["Wg"], w["h"], w["Np"][0], w["Np"][1],
                                               w["Ng"][0], w["Ng"][1], vertex_order="grid")
    rwg = m.build_rwg_interior({"V": V, "F": F})
    pe = m.pick_port_edge_by_point_and_layer(rwg, (0.0, -7e-3, +w["h"] / 2), +1)
    ge = m.pick_port_edge_by_point_and_layer(rwg, (0.0, -7e-3, -w["h"] / 2), -1)
    pre = m.efie_precompute_pack({"V": V, "F": F}, OPTS_REF_GPU)
    spread = 1.5 * float(np.mean(rwg["len"]))
    a, b, n = w["freqs"]
    freqs = np.linspace(a, b, n)
    args = [V, F, rwg["edge"], rwg["plusTri"], rwg["minusTri"], rwg["plusSign"], rwg["minusSign"], rwg["rp"],
            rwg["rm"], rwg["Ap"], rwg["Am"], rwg["len"], pre]
    tail = [MU0, EPS0, pe, ge, 1.0, spread, 50.0]
    return dict(V=V, F=F, rwg=rwg, pe=pe, ge=ge, pre=pre, spread=spread, freqs=freqs, args=args, tail=tail,
                Ne=rwg["Ne"], Nt=F.shape[0])


def _nbytes(objs):
    tot = 0
    for o in objs:
        if isinstance(o, dict):
            tot += _nbytes(list(o.values()))
        elif isinstance(o, np.ndarray):
            tot += o.nbytes
        else:
            tot += 8
    return tot


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def _traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def roofline(classes):
    """Roofline entry for the dominant kernel class (largest device time)."""
    peaks, src = _peaks()
    cand = {k: v for k, v in classes.items() if v["launches"] > 0 and v["ms"] > 0 and k != "other"}
    if not cand:
        return None
    name = max(cand, key=lambda k: cand[k]["ms"])
    c = cand[name]
    per_launch_ms = c["ms"] / c["launches"]
    per_launch_work = c["work"] / c["launches"]
    tr = _traffic().get(name)
    if name == "gemm":
        achieved = per_launch_work / (per_launch_ms * 1e-3) / 1e12
        peak = peaks["bf16_tflops_sustained"]
        out = dict(bound="tensor", unit="TFLOP/s", peak_source=src + " bf16 sustained")
    elif name in ("quad", "nearself"):
        # FP64 point-pair evaluations; reported against HBM only for the schema -- see DESIGN.md
        achieved = per_launch_work / (per_launch_ms * 1e-3) / 1e9
        peak = None
        out = dict(bound="fp64", unit="Gpair/s", peak_source="none")
    else:
        achieved = per_launch_work / (per_launch_ms * 1e-3) / 1e9
        peak = peaks["hbm_gbs"]
        out = dict(bound="hbm", unit="GB/s", peak_source=src)
    out.update(kernel=name, achieved=achieved, peak=peak, frac=(achieved / peak) if peak else None,
               traffic=tr, launches=c["launches"], ms_per_launch=per_launch_ms)
    return out


def cpu_baseline_sample(inp, n_points=1):
    """Oracle port of the reference CPU path on all host cores, one frequency point."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_c  # noqa: E402  (CPU-baseline leg only)
    oracle_c.build()
    rwg = dict(inp["rwg"])
    pre = inp["pre"]
    cores = os.cpu_count() or 1
    b = None
    t0 = time.perf_counter()
    for f in inp["freqs"][:n_points]:
        omega = 2 * math.pi * f
        k = omega * np.sqrt(MU0 * EPS0 + 0j)
        Z = oracle_c.assemble_z(rwg, pre, k, omega, MU0, EPS0, nthreads=cores)
        if b is None:
            m = _pkg()
            # RHS is O(Ne): reuse the product's host RHS through a tiny ggassemble-free path
            b = _rhs(inp)
        x = np.linalg.solve(Z, b)
        _ = np.sum(x)
    dt = time.perf_counter() - t0
    return n_points / dt, cores, dt


def _rhs(inp):
    V = inp["V"]
    E = inp["rwg"]["edge"].astype(np.int64) - 1
    c = 0.5 * (V[E[:, 0]] + V[E[:, 1]])
    zmid = 0.5 * (c[:, 2].min() + c[:, 2].max())
    lay = np.where(c[:, 2] > zmid, 1, -1)

    def w(e0):
        d = np.sqrt(((c - c[e0]) ** 2).sum(1))
        v = np.exp(-(d / inp["spread"]) ** 2) * (lay == lay[e0])
        return v / v.sum()
    return (0.5 * w(inp["pe"] - 1) - 0.5 * w(inp["ge"] - 1)).astype(np.complex128)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    m = _pkg()
    inp = build_inputs(m, args.workload)
    cores = os.cpu_count() or 1
    for _ in range(min(args.warmup, 1)):
        cpu_baseline_sample(inp, 1)
    times = []
    for _ in range(args.steps):
        v, cores, dt = cpu_baseline_sample(inp, 1)
        times.append(dt)
    value = args.steps / sum(times)
    line = dict(metric=METRIC, value=value, unit="freq points/s", impl="reference", n_gpus=args.gpus,
                steps=args.steps, warmup=min(args.warmup, 1), ms_per_step=1e3 * sum(times) / args.steps,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="c128", data="synthetic",
                config=dict(workload=args.workload, Ne=inp["Ne"], Nt=inp["Nt"], batch=1,
                            scheme="reference cached subdivision + softening (GPU option set)"),
                cpu_baseline=dict(value=value, unit="freq points/s", cores=cores, kind="port",
                                  sample="1 frequency point of %s per step: C restatement of CPU_FAST "
                                         "(OpenMP, %d threads) + numpy LAPACK solve" % (args.workload, cores)),
                e2e=dict(value=value, unit="freq points/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    # the reference's own CUDA sweep (compiled from its sources) on a bounded sample
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ref_mex  # noqa: E402
        import torch
        if torch.cuda.is_available():
            n = max(2, min(args.batch, 4))
            fr = inp["freqs"][:n]
            r = inp["rwg"]
            mex = ref_mex.RefMex("patch_sweep_fastquad_ref")
            call = lambda ff: mex.call(2, inp["V"], inp["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"],
                                       r["minusSign"], r["rp"], r["rm"], r["Ap"], r["Am"], r["len"], inp["pre"],
                                       np.asarray(ff, np.float64), MU0, complex(EPS0), float(inp["pe"]),
                                       float(inp["ge"]), 1.0, inp["spread"], 50.0)
            call(fr[:1])
            t0 = time.perf_counter()
            call(fr)
            dt = time.perf_counter() - t0
            line["ref_gpu"] = dict(value=n / dt, unit="freq points/s",
                                   sample="%d frequency points through the reference patch_sweep_fastquad_cuda "
                                          "(compiled for sm_100a against a fake mex shim)" % n)
    except Exception as e:  # noqa: BLE001
        line["ref_gpu"] = dict(unavailable=str(e)[:200])
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    m = _pkg()
    nat = importlib.import_module(PKG + "._native")
    nat.context(local)
    # a dedicated stream: the library launches on it and it can be graph-captured
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    nat.check(nat.lib().efie_ctx_set_stream(nat.context(local), stream.cuda_stream))
    inp = build_inputs(m, args.workload)
    freqs = inp["freqs"]
    B = args.batch or len(freqs)
    # frequency slots of the plan: automatic, but no more than the points of a step
    opts = m.sweep_opts(solver=args.solver, timing=False, scheme=args.scheme,
                        batch=B if B < 8 else 0, lu_nb=args.lu_nb)
    pargs = list(inp["args"])
    if args.scheme == "extract":
        pargs[-1] = None   # no prepack: the rule points come from the mesh
    plan = m.SweepPlan(*pargs, *inp["tail"], opts=opts, rule_order=RULE[args.scheme])

    def batch(step):
        # each rank sweeps its own frequency points (replicas)
        i0 = ((step * world + rank) * B) % len(freqs)
        idx = (np.arange(B) + i0) % len(freqs)
        return freqs[idx]

    for s in range(args.warmup):
        plan.run(batch(s))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches = 0
    fallback = 0
    relres = 0.0
    iters = 0
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for s in range(args.steps):
            plan.run(batch(args.warmup + s))
            st = plan.stats
            launches += st["n_launches"]
            fallback += st["n_fp64_fallback"]
            relres = max(relres, st["max_relres"])
            iters = max(iters, st["refine_iters_max"])
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_points = args.steps * B * world
    value = total_points / (ms * 1e-3)
    # per-class breakdown (roofline): one more step with CUDA events around
    # every launch (eager launches), outside the timed region
    plan.set_timing(True)
    plan.run(batch(args.warmup + args.steps))
    classes = {k: dict(v) for k, v in plan.stats["classes"].items()}
    plan.close()

    # e2e: the public API call with host arrays (upload + sweep + results) per step
    e2e_ms = []
    h2d = _nbytes(inp["args"]) + B * 8
    for s in range(max(1, args.steps)):
        fr = batch(args.warmup + s)
        t0 = time.perf_counter()
        if args.scheme == "ref":
            m.patch_sweep_fastquad_cuda(*inp["args"], fr, *inp["tail"], opts=m.sweep_opts(solver=args.solver, lu_nb=args.lu_nb))
        else:
            # plan create (host mesh upload) + run + destroy through the C ABI
            p2 = m.SweepPlan(*pargs, *inp["tail"], opts=m.sweep_opts(solver=args.solver, scheme="extract", lu_nb=args.lu_nb),
                             rule_order=RULE[args.scheme])
            p2.run(fr)
            p2.close()
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e = sum(e2e_ms)
    if dist:
        t = torch.tensor([e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = float(t.item())
    e2e_value = (max(1, args.steps) * B * world) / (e2e * 1e-3)

    line = None
    if rank == 0:
        line = dict(metric=METRIC, value=value, unit="freq points/s", n_gpus=world, steps=args.steps,
                    warmup=args.warmup, ms_per_step=ms / args.steps, higher_is_better=True, scaling="weak",
                    vs_baseline=None, dtype="c128 (assembly, residual) / c64 (LU)" if args.solver == "mixed"
                    else "c128", data="synthetic",
                    config=dict(workload=args.workload, Ne=inp["Ne"], Nt=inp["Nt"], batch=B,
                                solver=args.solver, parallelism="replicas x%d" % world,
                                scheme=SCHEME_NAME[args.scheme],
                                l2="working set per step > L2 (Z c128 %.0f MB)" % (16e-6 * inp["Ne"] ** 2)),
                    e2e=dict(value=e2e_value, unit="freq points/s", h2d_bytes_per_step=h2d,
                             d2h_bytes_per_step=2 * 16 * B),
                    gpu_launches=launches, clocks=clk.summary(),
                    accuracy=dict(max_relres=relres, refine_iters_max=iters, fp64_fallbacks=fallback),
                    roofline=roofline(classes),
                    phases_ms_per_point={k: v["ms"] / B for k, v in classes.items()},
                    phases_note="one extra step with per-launch CUDA events (eager launches), outside the "
                                "timed region; the timed steps replay the factorization as a CUDA graph")
        if world == 1 and not args.no_cpu_baseline:
            v, cores, dt = cpu_baseline_sample(inp, 1)
            line["cpu_baseline"] = dict(value=v, unit="freq points/s", cores=cores, kind="port",
                                        sample="1 frequency point of %s: C restatement of CPU_FAST (OpenMP, %d "
                                               "threads) + numpy LAPACK solve, %.1f s" % (args.workload, cores, dt))
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _family():
    sur = importlib.import_module(PKG + ".surrogate")
    return sur, sur.sample_designs(FAMILY["n"], seed=FAMILY["seed"], pitch=FAMILY["pitch"],
                                   ground_pitch=FAMILY["ground_pitch"])


def run_family(args):
    """cfg3: one step = one design of the family (host mesh -> plan -> 41-point
    sweep -> results); designs of uneven Ne, each swept with batched
    frequencies.  Device time (CUDA events on the library's stream) covers
    geometry upload, assembly, solve and port reduction; e2e adds the host
    producers and the result read-back (wall clock)."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    nat = importlib.import_module(PKG + "._native")
    nat.context(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    nat.check(nat.lib().efie_ctx_set_stream(nat.context(local), stream.cuda_stream))
    sur, designs = _family()
    nf = FAMILY["nfreq"]

    def step(i):
        d = designs[(i * world + rank) % len(designs)]
        x = sur.design_inputs(d)
        plan = sur.design_plan(d, inputs=x)
        Zin, _ = plan.run(d.band(nf))
        plan.close()
        return x["Ne"], Zin

    for i in range(args.warmup):
        step(i)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    Ns = []
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        ev0.record(stream)
        for i in range(args.steps):
            n, _ = step(args.warmup + i)
            Ns.append(n)
        ev1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms, wall * 1e3], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, wall = float(t[0].item()), float(t[1].item()) * 1e-3
    pts = args.steps * nf * world
    if rank == 0:
        line = dict(metric=METRIC, value=pts / (ms * 1e-3), unit="freq points/s", n_gpus=world, steps=args.steps,
                    warmup=args.warmup, ms_per_step=ms / args.steps, higher_is_better=True, scaling="weak",
                    vs_baseline=None, dtype="c128 (assembly, residual) / c64 (LU)", data="synthetic",
                    config=dict(workload="cfg3", designs=FAMILY["n"], Ne_of_timed_designs=Ns, freqs_per_design=nf,
                                mesh_pitch_mm=[1e3 * FAMILY["pitch"], 1e3 * FAMILY["ground_pitch"]],
                                scheme="Dunavant 7-point rule + analytic 1/R extraction", solver="mixed (GMRES)",
                                parallelism="replicas x%d" % world),
                    e2e=dict(value=pts / wall, unit="freq points/s", h2d_bytes_per_step=None,
                             d2h_bytes_per_step=nf * 32),
                    clocks=clk.summary())
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_surrogate(args):
    """cfg4: train the surrogate on solver samples of the design family, then
    locate the |S11| minimum of held-out designs with surrogate-guided
    adaptive sweeps and with dense 201-point sweeps."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    sur, _ = _family()
    nper = 40
    ntrain = max(1, args.samples // nper)
    train = sur.sample_designs(ntrain, seed=11, pitch=FAMILY["pitch"], ground_pitch=FAMILY["ground_pitch"])
    t0 = time.perf_counter()
    X, T = sur.generate_samples(train, nper, seed=12)
    t_data = time.perf_counter() - t0
    net = sur.Surrogate(seed=13)
    t0 = time.perf_counter()
    hist = net.train(X, T, epochs=args.epochs, batch=1024, lr=2e-3)
    hist2 = net.train(X, T, epochs=max(1, args.epochs // 3), batch=1024, lr=3e-4)
    t_train = time.perf_counter() - t0
    test = sur.sample_designs(max(3, args.steps), seed=99, pitch=FAMILY["pitch"], ground_pitch=FAMILY["ground_pitch"])
    rows = []
    t_ad = t_dn = t_un = 0.0
    for d in test:
        plan = sur.design_plan(d)
        plan.run(d.band(8))     # warm the plan
        t0 = time.perf_counter()
        dn = sur.dense_sweep(d, 201, plan)
        t_dn += time.perf_counter() - t0
        t0 = time.perf_counter()
        ad = sur.adaptive_sweep(d, net, plan)
        t_ad += time.perf_counter() - t0
        t0 = time.perf_counter()
        un = sur.uniform_sweep_estimate(d, ad["solves"], plan)
        t_un += time.perf_counter() - t0
        step = (d.band(201)[1] - d.band(201)[0])
        rows.append(dict(Ne=plan.Ne, solves=ad["solves"], rounds=ad["rounds"], fallback=ad["fallback"],
                         fmin_err_steps=abs(ad["f_min"] - dn["f_min"]) / step,
                         uniform_err_steps=abs(un["f_min"] - dn["f_min"]) / step))
        plan.close()
    nd = len(test)
    solves = sum(r["solves"] for r in rows)
    line = dict(metric=METRIC, value=201 * nd / t_ad, unit="dense-equivalent freq points/s", n_gpus=1,
                steps=nd, warmup=1, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="c128/c64 solver; MLP bf16 weights, fp32 accumulate", data="synthetic",
                config=dict(workload="cfg4", train_samples=int(len(X)), train_designs=ntrain, epochs=args.epochs,
                            mlp="5 -> 4 x 256 SiLU -> 3 (log|Zin|, cos, sin arg Zin)", test_designs=nd),
                surrogate=dict(data_s=t_data, solver_samples_per_s=len(X) / t_data, train_s=t_train,
                               loss_first=float(hist[0]), loss_last=float(hist2[-1]),
                               adaptive_solves_per_design=solves / nd,
                               adaptive_solved_points_per_s=solves / t_ad,
                               dense_points_per_s=201 * nd / t_dn,
                               fmin_err_steps_max=max(r["fmin_err_steps"] for r in rows),
                               fmin_err_steps_mean=statistics.mean(r["fmin_err_steps"] for r in rows),
                               uniform_same_budget_err_steps_mean=statistics.mean(r["uniform_err_steps"]
                                                                                  for r in rows),
                               fallbacks=sum(1 for r in rows if r["fallback"]), designs=rows),
                e2e=dict(value=201 * nd / t_ad, unit="dense-equivalent freq points/s", h2d_bytes_per_step=None,
                         d2h_bytes_per_step=None))
    print(json.dumps(line), flush=True)
    net.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS) + ["cfg3", "cfg4"], default="cfg2")
    ap.add_argument("--samples", type=int, default=20000, help="cfg4: solver samples for training")
    ap.add_argument("--epochs", type=int, default=300, help="cfg4: training epochs")
    ap.add_argument("--batch", type=int, default=0, help="frequency points per step (0 = the whole sweep)")
    ap.add_argument("--solver", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--lu-nb", type=int, default=0, choices=[0, 64, 128, 256, 512],
                    help="outer LU panel width (0: the library's choice)")
    ap.add_argument("--scheme", choices=["ref", "extract"], default="ref",
                    help="ref: the reference's cached subdivision + softening; extract: Dunavant 7-point rule "
                         "+ analytic 1/R extraction")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if args.workload in ("cfg3", "cfg4"):
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no design-family or "
                              "surrogate sweep; its CPU path is timed on the single-design workloads"}))
            return 0
        return run_reference(args)
    if args.workload == "cfg3":
        return run_family(args)
    if args.workload == "cfg4":
        return run_surrogate(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
