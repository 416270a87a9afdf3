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
its sources, oracle/_ref) on a bounded sample as ``ref_gpu``.  Its inputs
(mesh, RWG numbering, ports, prepack) come from the oracle's restatement of
the MATLAB producers, so that process loads no library of this package.

The default line (cfg2) also carries the plain FP64 GPU path of this package
(complex128 assembly + cuSOLVER Zgetrf/Zgetrs) on the same frequency points
as ``fp64_gpu``, the Zin error of every point against it and of sampled
points against the CPU oracle, and a ``secondary`` block: cfg2 with the
Dunavant 7-point rule + analytic extraction, and cfg5 (Ne 19936) on a few
points, each with its Zin error against the FP64 path.
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


# FP64 operations the assembly's pipes execute per point-pair evaluation and
# frequency (QPE) of the regular-pair kernel: DADD + DMUL + 2 DFMA from the
# sass instruction counters of one captured launch of the four-frequency
# kernel (cfg2), divided by the launch's QPE.  The transcendental functions
# (sqrt, sincos, the reciprocal) are FP64 instruction sequences, so this is
# the work the FP64 pipe does per QPE, not a textbook flop count; it is kept
# in profiles/traffic.json beside the DRAM bytes of the same capture.
FP64_OPS_PER_QPE = None


def _fp64_ops_per_qpe():
    tr = _traffic().get("quad_fp64_ops_per_qpe")
    return float(tr) if tr else FP64_OPS_PER_QPE


def _fp64_peak_tflops():
    """Measured FP64 throughput of cuBLAS DGEMM (torch float64 matmul) on this GPU."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    reps = 5
    for _ in range(reps):
        torch.matmul(a, b)
    e1.record()
    torch.cuda.synchronize()
    tf = reps * 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12
    del a, b
    torch.cuda.empty_cache()
    return tf


def roofline(classes, name=None, fp64_peak=None):
    """Roofline entry for one kernel class (default: the dominant one, by device time)."""
    peaks, src = _peaks()
    cand = {k: v for k, v in classes.items() if v["launches"] > 0 and v["ms"] > 0 and k != "other"}
    if not cand:
        return None
    if name is None:
        name = max(cand, key=lambda k: cand[k]["ms"])
    if name not in cand:
        return None
    c = cand[name]
    per_launch_ms = c["ms"] / c["launches"]
    per_launch_work = c["work"] / c["launches"]
    tr = _traffic().get(name)
    if name == "gemm":
        achieved = per_launch_work / (per_launch_ms * 1e-3) / 1e12
        peak = peaks["bf16_tflops_sustained"]
        out = dict(bound="tensor", unit="TFLOP/s", peak_source=src + " bf16 sustained")
    elif name == "quad":
        # QPE/s times the FP64 operations per QPE, against measured DGEMM
        ops = _fp64_ops_per_qpe()
        qpe_rate = per_launch_work / (per_launch_ms * 1e-3)
        achieved = qpe_rate * ops / 1e12 if ops else None
        peak = fp64_peak
        out = dict(bound="fp64", unit="TFLOP/s", peak_source="measured cuBLAS DGEMM (torch float64 matmul)",
                   gqpe_per_s=qpe_rate / 1e9, fp64_ops_per_qpe=ops)
    else:
        achieved = per_launch_work / (per_launch_ms * 1e-3) / 1e9
        peak = peaks["hbm_gbs"]
        out = dict(bound="hbm", unit="GB/s", peak_source=src)
    out.update(kernel=name, achieved=achieved, peak=peak,
               frac=(achieved / peak) if (peak and achieved is not None) else None,
               traffic=tr, launches=c["launches"], ms_per_launch=per_launch_ms)
    return out


def _oracle_mod():
    """The oracle package (test infrastructure): checker and CPU baseline only."""
    d = os.path.join(ROOT, "oracle")
    if d not in sys.path:
        sys.path.insert(0, d)
    import efie_oracle  # noqa: E402
    import oracle_c  # noqa: E402
    return efie_oracle, oracle_c


def oracle_inputs(wl):
    """Mesh, RWG, ports, prepack and RHS of a workload through the oracle's
    restatement of the MATLAB producers (no library of this package)."""
    eo, _ = _oracle_mod()
    w = WORKLOADS[wl]
    a, b, n = w["freqs"]
    d = eo.Design(Lp=w["Lp"], Wp=w["Wp"], Lg=w["Lg"], Wg=w["Wg"], h=w["h"], Np_x=w["Np"][0], Np_y=w["Np"][1],
                  Ng_x=w["Ng"][0], Ng_y=w["Ng"][1], feed=(0.0, -7e-3), mu=MU0, eps=EPS0, V0=1.0, Z0=50.0,
                  freqs=np.linspace(a, b, n), vertex_order="grid", opts=dict(OPTS_REF_GPU))
    return eo.build_problem(d)


def cpu_oracle_points(prob, freqs):
    """The reference CPU path per frequency point, restated in the oracle:
    CPU_FAST assembly (C, OpenMP, all host cores) + LAPACK solve + Zin.
    Returns (Zin [n], seconds, cores)."""
    eo, oc = _oracle_mod()
    oc.build()
    d = prob["design"]
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    Zin = np.zeros(len(freqs), np.complex128)
    for i, f in enumerate(freqs):
        omega, k, _, _ = eo.physics(f, d.mu, d.eps)
        Z = oc.assemble_z(prob["rwg"], prob["prepack"], k, omega, d.mu, d.eps, nthreads=cores)
        x = np.linalg.solve(Z, prob["b"].astype(np.complex128))
        Zin[i], _ = eo.zin_s11(eo.port_current(x, prob["wP"], prob["wG"], prob["rwg"]["len"]), d.V0, d.Z0)
    return Zin, time.perf_counter() - t0, cores


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    prob = oracle_inputs(args.workload)
    freqs = prob["design"].freqs
    for _ in range(min(args.warmup, 1)):
        cpu_oracle_points(prob, freqs[:1])
    times = []
    cores = os.cpu_count() or 1
    for s in range(args.steps):
        _, dt, cores = cpu_oracle_points(prob, freqs[s % len(freqs):s % len(freqs) + 1])
        times.append(dt)
    value = args.steps / sum(times)
    line = dict(metric=METRIC, value=value, unit="freq points/s", impl="reference", n_gpus=args.gpus,
                steps=args.steps, warmup=min(args.warmup, 1), ms_per_step=1e3 * sum(times) / args.steps,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="c128", data="synthetic",
                config=dict(workload=args.workload, Ne=prob["rwg"]["Ne"], Nt=int(prob["F"].shape[0]), batch=1,
                            scheme="reference cached subdivision + softening (GPU option set)",
                            inputs="oracle restatement of the MATLAB producers"),
                cpu_baseline=dict(value=value, unit="freq points/s", cores=cores, kind="port",
                                  sample="1 frequency point of %s per step: C restatement of CPU_FAST "
                                         "(OpenMP, %d threads) + numpy LAPACK solve" % (args.workload, cores)),
                e2e=dict(value=value, unit="freq points/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    # the reference's own CUDA sweep (compiled from its sources) on a bounded sample
    try:
        import ref_mex  # noqa: E402  (oracle/, on sys.path through _oracle_mod)
        import torch
        if torch.cuda.is_available():
            n = max(8, min(args.batch or 8, 16))
            fr = freqs[:n]
            ref_mex.patch_sweep_fastquad(prob, fr[:1])
            t0 = time.perf_counter()
            ref_mex.patch_sweep_fastquad(prob, fr)
            dt = time.perf_counter() - t0
            line["ref_gpu"] = dict(value=n / dt, unit="freq points/s",
                                   sample="%d frequency points through the reference patch_sweep_fastquad_cuda "
                                          "(compiled for sm_100a against a fake mex shim)" % n)
    except Exception as e:  # noqa: BLE001
        line["ref_gpu"] = dict(unavailable=str(e)[:200])
    print(json.dumps(line), flush=True)
    return 0


def _stream_time(stream, fn):
    """Device time (ms, CUDA events on `stream`) of fn() and its result."""
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


def _rel(a, b):
    return float(np.max(np.abs(a - b) / np.abs(b))) if len(b) else None


def fp64_arm(m, pargs, tail, freqs, stream, scheme="ref"):
    """The plain FP64 GPU path (complex128 assembly + cuSOLVER Zgetrf/Zgetrs
    per frequency) on `freqs`: (points/s, Zin)."""
    plan = m.SweepPlan(*pargs, *tail, opts=m.sweep_opts(solver="fp64", scheme=scheme), rule_order=RULE[scheme])
    plan.run(freqs[:2])
    ms, (Zin, _) = _stream_time(stream, lambda: plan.run(freqs))
    plan.close()
    return len(freqs) / (ms * 1e-3), Zin


def secondary_block(m, stream):
    """cfg2 with the benchmark configuration's own quadrature (Dunavant 7-point
    rule + analytic extraction) on all 101 points, and cfg5 (Ne 19936) on 8 points: points/s
    of the mixed solver and Zin error against the FP64 GPU path."""
    out = {}
    inp = build_inputs(m, "cfg2")
    pargs = list(inp["args"])
    pargs[-1] = None
    fr = inp["freqs"]
    plan = m.SweepPlan(*pargs, *inp["tail"], opts=m.sweep_opts(scheme="extract"), rule_order=RULE["extract"])
    plan.run(fr[:4])
    plan.run(fr)
    ms, (Zin, _) = _stream_time(stream, lambda: plan.run(fr))
    st = plan.stats
    plan.close()
    v64, Z64 = fp64_arm(m, pargs, inp["tail"], fr, stream, scheme="extract")
    out["cfg2_extract"] = dict(value=len(fr) / (ms * 1e-3), unit="freq points/s", points=len(fr), Ne=inp["Ne"],
                               scheme=SCHEME_NAME["extract"], fp64_gpu=v64,
                               max_rel_zin_err_vs_fp64=_rel(Zin, Z64), max_relres=st["max_relres"],
                               refine_iters_max=st["refine_iters_max"], fp64_fallbacks=st["n_fp64_fallback"])
    inp = build_inputs(m, "cfg5")
    fr = inp["freqs"][::7][:8]
    # plan creation from the host prepack (host producers + upload + near-pair
    # scan), then with the prepack computed on the device from V/F
    t0 = time.perf_counter()
    pre = m.efie_precompute_pack({"V": inp["V"], "F": inp["F"]}, OPTS_REF_GPU)
    plan = m.SweepPlan(*inp["args"][:-1], pre, *inp["tail"], opts=m.sweep_opts(), rule_order=0)
    t_host = time.perf_counter() - t0
    plan.close()
    del pre
    t0 = time.perf_counter()
    plan = m.SweepPlan(*inp["args"][:-1], None, *inp["tail"], opts=m.sweep_opts(), precompute=OPTS_REF_GPU)
    t_plan = time.perf_counter() - t0
    plan.run(fr[:2])
    ms, (Zin, _) = _stream_time(stream, lambda: plan.run(fr))
    st = plan.stats
    plan.close()
    f3 = fr[[0, 3, 7]]
    v64, Z64 = fp64_arm(m, inp["args"], inp["tail"], f3, stream)
    out["cfg5"] = dict(value=len(fr) / (ms * 1e-3), unit="freq points/s", points=len(fr), Ne=inp["Ne"],
                       scheme=SCHEME_NAME["ref"], plan_create_s=dict(host_prepack=t_host, device_prepack=t_plan),
                       fp64_gpu=v64, fp64_points=len(f3),
                       max_rel_zin_err_vs_fp64=_rel(Zin[[0, 3, 7]], Z64), max_relres=st["max_relres"],
                       refine_iters_max=st["refine_iters_max"], fp64_fallbacks=st["n_fp64_fallback"])
    return out


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
    # tensor-core tile widths: the command line's, else the autotuner's table
    tuned = importlib.import_module(PKG + ".autotune").tuned_opts(inp["Ne"])
    tiles = (args.tile_chain or (tuned[2] if tuned else 0), args.tile_bulk or (tuned[3] if tuned else 0))
    resident = (args.resident_chain if args.resident_chain >= 0 else (tuned[4] if tuned else 0),
                args.resident_bulk if args.resident_bulk >= 0 else (tuned[5] if tuned else 0))
    opts = m.sweep_opts(solver=args.solver, timing=False, scheme=args.scheme,
                        batch=B if B < 8 else 0, lu_nb=args.lu_nb, tile_chain=tiles[0], tile_bulk=tiles[1],
                        resident_chain=resident[0], resident_bulk=resident[1], nfreq_hint=B,
                        share_factors=args.share_factors)
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
    shared = 0
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for s in range(args.steps):
            fr_last = batch(args.warmup + s)
            Zin_last, _ = plan.run(fr_last)
            st = plan.stats
            launches += st["n_launches"]
            fallback += st["n_fp64_fallback"]
            relres = max(relres, st["max_relres"])
            iters = max(iters, st["refine_iters_max"])
            shared += st["n_shared_factors"]
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

    # e2e: the public API call with host arrays (upload + sweep + results) per
    # step, after one untimed call (the first call after the resident plan's
    # release refills the device pool)
    e2e_ms = []
    h2d = _nbytes(inp["args"]) + B * 8

    def e2e_call(fr):
        if args.scheme == "ref":
            m.patch_sweep_fastquad_cuda(*inp["args"], fr, *inp["tail"],
                                        opts=m.sweep_opts(solver=args.solver, lu_nb=args.lu_nb, tile_chain=tiles[0],
                                                          tile_bulk=tiles[1], resident_chain=resident[0],
                                                          resident_bulk=resident[1],
                                                          share_factors=args.share_factors))
        else:
            # plan create (host mesh upload) + run + destroy through the C ABI
            p2 = m.SweepPlan(*pargs, *inp["tail"],
                             opts=m.sweep_opts(solver=args.solver, scheme="extract", lu_nb=args.lu_nb,
                                               tile_chain=tiles[0], tile_bulk=tiles[1], resident_chain=resident[0],
                                               resident_bulk=resident[1], nfreq_hint=B,
                                               share_factors=args.share_factors),
                             rule_order=RULE[args.scheme])
            p2.run(fr)
            p2.close()

    e2e_call(batch(args.warmup))
    for s in range(max(1, args.steps)):
        fr = batch(args.warmup + s)
        t0 = time.perf_counter()
        e2e_call(fr)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e = sum(e2e_ms)
    if dist:
        t = torch.tensor([e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = float(t.item())
    e2e_value = (max(1, args.steps) * B * world) / (e2e * 1e-3)

    # the metric's FP64 arm: the plain FP64 GPU path on the same points, and
    # the Zin error of every point of the last timed step against it
    fp64 = None
    accuracy = dict(max_relres=relres, refine_iters_max=iters, fp64_fallbacks=fallback,
                    points_on_shared_factors=shared, points_timed=args.steps * B)
    if args.solver == "mixed" and not args.no_fp64_arm:
        v64, Z64 = fp64_arm(m, pargs, inp["tail"], fr_last, stream, scheme=args.scheme)
        fp64 = dict(value=v64, unit="freq points/s", points=len(fr_last),
                    solver="complex128 assembly + cuSOLVER Zgetrf/Zgetrs per frequency")
        err = np.abs(Zin_last - Z64) / np.abs(Z64)
        accuracy.update(max_rel_zin_err_vs_fp64=float(err.max()), median_rel_zin_err_vs_fp64=float(np.median(err)),
                        points_vs_fp64=len(err))
    fp64_peak = None
    if rank == 0:
        try:
            fp64_peak = _fp64_peak_tflops()
        except Exception:  # noqa: BLE001
            fp64_peak = None
    secondary = None
    if rank == 0 and world == 1 and args.workload == "cfg2" and args.scheme == "ref" and not args.no_secondary:
        secondary = secondary_block(m, stream)

    line = None
    if rank == 0:
        line = dict(metric=METRIC, value=value, unit="freq points/s", n_gpus=world, steps=args.steps,
                    warmup=args.warmup, ms_per_step=ms / args.steps, higher_is_better=True, scaling="weak",
                    vs_baseline=None, dtype="c128 (assembly, residual) / c64 (LU)" if args.solver == "mixed"
                    else "c128", data="synthetic",
                    config=dict(workload=args.workload, Ne=inp["Ne"], Nt=inp["Nt"], batch=B,
                                solver=args.solver, parallelism="replicas x%d" % world,
                                tc_tiles="256x%s (panel chain) / 256x%s (outer panels)"
                                         % ("128 resident" if resident[0] else tiles[0] or 256,
                                            "128 resident" if resident[1] else tiles[1] or 256),
                                scheme=SCHEME_NAME[args.scheme],
                                share_factors=(args.share_factors or "auto") if args.solver == "mixed" else 1,
                                l2="working set per step > L2 (Z c128 %.0f MB)" % (16e-6 * inp["Ne"] ** 2)),
                    e2e=dict(value=e2e_value, unit="freq points/s", h2d_bytes_per_step=h2d,
                             d2h_bytes_per_step=2 * 16 * B, ms_per_step=[round(x, 2) for x in e2e_ms]),
                    gpu_launches=launches, clocks=clk.summary(),
                    accuracy=accuracy, fp64_gpu=fp64,
                    roofline=roofline(classes),
                    roofline_assembly=roofline(classes, "quad", fp64_peak),
                    roofline_tensor=roofline(classes, "gemm"),
                    # the HBM-bound classes: algorithmic bytes over their event time
                    roofline_hbm={k: roofline(classes, k) for k in ("trsv", "residual", "gather")},
                    phases_ms_per_point={k: v["ms"] / B for k, v in classes.items()},
                    phases_note="one extra step with per-launch CUDA events (eager launches, the LU's "
                                "look-ahead stream folded into the chain's so each pair of events brackets "
                                "one kernel running alone), outside the timed region; the timed steps replay "
                                "the factorization as a CUDA graph with the look-ahead")
        if world == 1 and not args.no_cpu_baseline:
            # the oracle's CPU path on the box's host cores: the first point of
            # the last step and the point furthest from the FP64 arm
            prob = oracle_inputs(args.workload) if args.scheme == "ref" else None
            if prob is not None:
                j = [0]
                if "max_rel_zin_err_vs_fp64" in accuracy:
                    j.append(int(np.argmax(np.abs(Zin_last - Z64) / np.abs(Z64))))
                j = sorted(set(j))
                Zc, dt, cores = cpu_oracle_points(prob, fr_last[j])
                line["cpu_baseline"] = dict(value=len(j) / dt, unit="freq points/s", cores=cores, kind="port",
                                            sample="%d frequency point(s) of %s: C restatement of CPU_FAST (OpenMP, "
                                                   "%d threads) + numpy LAPACK solve, %.1f s"
                                                   % (len(j), args.workload, cores, dt))
                accuracy.update(max_rel_zin_err_vs_cpu_oracle=_rel(Zin_last[j], Zc), points_vs_cpu_oracle=len(j))
        if secondary:
            line["secondary"] = secondary
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
    """cfg3: one step = ``--designs`` designs of the family (GPU mesh + RWG ->
    plan -> 41-point sweep -> results), ``--workers`` of them in flight at
    once on their own contexts and streams (surrogate.sweep_family).  Device
    time: CUDA events on a root stream that every worker stream waits on at
    the start and that waits on every worker stream at the end; it covers
    mesh building, plan set-up, assembly, solve and port reduction and the
    host work between them.  e2e adds the Python driver around it (wall
    clock)."""
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
    sur, designs = _family()
    nf = FAMILY["nfreq"]
    W, D = max(1, args.workers), max(1, args.designs)
    root = torch.cuda.Stream()
    streams = [torch.cuda.Stream() for _ in range(W)]

    def chunk(i):
        # the D designs of step i for this rank (ranks take disjoint designs)
        return [designs[((i * world + rank) * D + j) % len(designs)] for j in range(D)]

    times = []

    def step(i):
        out = sur.sweep_family(chunk(i), nf, workers=W, device=local, streams=[st.cuda_stream for st in streams],
                               times=times)
        return [n for n, _ in out]

    for i in range(args.warmup):
        step(i)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    times.clear()
    Ns = []
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        ev0.record(root)
        for st in streams:
            st.wait_event(ev0)
        for i in range(args.steps):
            Ns += step(args.warmup + i)
        for st in streams:
            e = torch.cuda.Event()
            e.record(st)
            root.wait_event(e)
        ev1.record(root)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms, wall * 1e3], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, wall = float(t[0].item()), float(t[1].item()) * 1e-3
    pts = args.steps * D * nf * world
    if rank == 0:
        line = dict(metric=METRIC, value=pts / (ms * 1e-3), unit="freq points/s", n_gpus=world, steps=args.steps,
                    warmup=args.warmup, ms_per_step=ms / args.steps, higher_is_better=True, scaling="weak",
                    vs_baseline=None, dtype="c128 (assembly, residual) / c64 (LU)", data="synthetic",
                    config=dict(workload="cfg3", designs=FAMILY["n"], designs_per_step=D, workers=W,
                                Ne_of_timed_designs=Ns, freqs_per_design=nf,
                                mesh_pitch_mm=[1e3 * FAMILY["pitch"], 1e3 * FAMILY["ground_pitch"]],
                                scheme="Dunavant 7-point rule + analytic 1/R extraction", solver="mixed (GMRES)",
                                mesh="built on the GPU (mesh, RWG numbering, ports)",
                                parallelism="replicas x%d, %d designs in flight per GPU" % (world, W)),
                    e2e=dict(value=pts / wall, unit="freq points/s", h2d_bytes_per_step=None,
                             d2h_bytes_per_step=D * nf * 32),
                    plan_create_s_per_design=statistics.mean(t for t, _ in times) if times else None,
                    sweep_s_per_design=statistics.mean(t for _, t in times) if times else None,
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
    ap.add_argument("--workers", type=int, default=3, help="cfg3: designs in flight at once per GPU")
    ap.add_argument("--designs", type=int, default=8, help="cfg3: designs per step")
    ap.add_argument("--epochs", type=int, default=300, help="cfg4: training epochs")
    ap.add_argument("--batch", type=int, default=0, help="frequency points per step (0 = the whole sweep)")
    ap.add_argument("--solver", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--lu-nb", type=int, default=0, choices=[0, 64, 128, 256, 512],
                    help="outer LU panel width (0: the library's choice)")
    ap.add_argument("--scheme", choices=["ref", "extract"], default="ref",
                    help="ref: the reference's cached subdivision + softening; extract: Dunavant 7-point rule "
                         "+ analytic 1/R extraction")
    ap.add_argument("--tile-chain", type=int, default=0, choices=[0, 128, 256],
                    help="tensor-core tile width of the LU's K = 64 updates (0: the autotuner's table)")
    ap.add_argument("--tile-bulk", type=int, default=0, choices=[0, 128, 256],
                    help="tensor-core tile width of the outer panels' updates (0: the autotuner's table)")
    ap.add_argument("--resident-chain", type=int, default=-1, choices=[-1, 0, 1],
                    help="1: the LU's K = 64 updates on resident, pipelined CTA pairs (-1: the autotuner's table)")
    ap.add_argument("--share-factors", type=int, default=0,
                    help="mixed solver: factor only the first of each group of this many coarse-to-fine batches; "
                         "the others refine with their nearest neighbours' factors (1: factor every frequency, "
                         "0: the library's automatic choice)")
    ap.add_argument("--resident-bulk", type=int, default=-1, choices=[-1, 0, 1],
                    help="1: the LU's outer-panel updates on resident, pipelined CTA pairs (-1: the autotuner's "
                         "table)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-arm", action="store_true", help="skip the plain FP64 GPU path on the same points")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the extraction-scheme and cfg5 block of the default line")
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
