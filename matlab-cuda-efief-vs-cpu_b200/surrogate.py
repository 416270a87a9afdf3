"""Surrogate-guided adaptive frequency sweeps for families of patch designs.

No counterpart in the reference (its drivers sweep a fixed frequency list).
Pieces:

* ``PatchDesign`` / ``sample_designs``: parametric patch-over-ground designs
  (W, L, h, feed offset) meshed with the library's own producers;
* ``Surrogate``: the MLP of ``csrc/surrogate.cu`` (CUDA forward, backward and
  Adam; C ABI ``efie_mlp_*``) from normalised (W, L, h, feed, f) to
  (log|Zin/Z_SCALE|, cos arg Zin, sin arg Zin), a target whose error is a
  relative error of Zin at every magnitude;
* ``generate_samples``: training data from the EFIE solver itself;
* ``adaptive_sweep``: the surrogate proposes where the |S11| minimum is, the
  EFIE solver checks batches of points there, and the surrogate corrected by
  the solved points interpolates between them.  Solved values always win: the
  surrogate only places points and fills the gaps, and a sweep whose corrected
  surrogate still misses the solver by more than ``tol`` after ``max_rounds``
  falls back to the dense plain sweep.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _native as nat
from .api import (SweepPlan, build_patch_design_gpu, build_rwg_interior, make_patch_with_ground_mesh,
                  pick_port_edge_by_point_and_layer, sweep_opts)

MU0 = 4.0 * math.pi * 1e-7
C0 = 299792458.0
EPS0 = 1.0 / (MU0 * C0 * C0)
Z_SCALE = 50.0        # |Zin| is learned as log(|Zin| / Z_SCALE)
N_OUT = 3             # log|Zin|, cos(arg Zin), sin(arg Zin)
BAND = 0.2            # sweeps cover f0 (1 +- BAND), f0 = c / (2 L)


# ---------------------------------------------------------------------------
# Designs
# ---------------------------------------------------------------------------
@dataclass
class PatchDesign:
    """A patch W x L (x, y) at height h over a square ground plate of side
    ground_factor * max(W, L), fed at (0, feed) on the patch centreline."""
    W: float
    L: float
    h: float
    feed: float
    pitch: float = 2.5e-3          # patch mesh pitch
    ground_pitch: float = 5e-3     # ground mesh pitch
    ground_factor: float = 1.6

    @property
    def f0(self):
        return C0 / (2.0 * self.L)

    def band(self, n):
        return np.linspace(self.f0 * (1 - BAND), self.f0 * (1 + BAND), n)

    def cells(self):
        G = self.ground_factor * max(self.W, self.L)
        ng = max(2, int(round(G / self.ground_pitch)))
        return (max(2, int(round(self.W / self.pitch))), max(2, int(round(self.L / self.pitch))), ng, ng)


def sample_designs(n, seed=0, W=(25e-3, 45e-3), L=(20e-3, 40e-3), h=(0.8e-3, 3.2e-3), feed_frac=1.0 / 3.0,
                   pitch=2.5e-3, ground_pitch=5e-3):
    """n designs with W, L, h uniform in the given ranges and the feed offset
    uniform within +-feed_frac * L along the centreline."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        w = rng.uniform(*W)
        l = rng.uniform(*L)
        hh = rng.uniform(*h)
        fd = rng.uniform(-feed_frac, feed_frac) * l
        out.append(PatchDesign(w, l, hh, fd, pitch, ground_pitch))
    return out


def design_inputs(d: PatchDesign, device=True, ctx=None):
    """Mesh, RWG and port edges of a design (grid vertex order): built on the
    GPU (build_patch_design_gpu) or by the host producers; the two are
    bit-identical."""
    npx, npy, ngx, ngy = d.cells()
    G = d.ground_factor * max(d.W, d.L)
    if device:
        V, F, rwg, pe, ge = build_patch_design_gpu(d.L, d.W, G, G, d.h, npx, npy, ngx, ngy, feed=(0.0, d.feed),
                                                   vertex_order="grid", ctx=ctx)
    else:
        V, F, _, _ = make_patch_with_ground_mesh(d.L, d.W, G, G, d.h, npx, npy, ngx, ngy, vertex_order="grid")
        rwg = build_rwg_interior({"V": V, "F": F})
        pe = pick_port_edge_by_point_and_layer(rwg, (0.0, d.feed, +d.h / 2), +1)
        ge = pick_port_edge_by_point_and_layer(rwg, (0.0, d.feed, -d.h / 2), -1)
    spread = 1.5 * float(np.mean(rwg["len"]))
    return dict(V=V, F=F, rwg=rwg, pe=pe, ge=ge, spread=spread, Ne=rwg["Ne"])


def design_plan(d: PatchDesign, solver="mixed", batch=0, inputs=None, ctx=None, graphs=True, nfreq=0):
    """A SweepPlan of the design: Dunavant 7-point rule + analytic 1/R extraction
    (``nfreq``: the points its sweeps will solve, to size the batches)."""
    x = inputs or design_inputs(d, ctx=ctx)
    r = x["rwg"]
    return SweepPlan(x["V"], x["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"],
                     r["rm"], r["Ap"], r["Am"], r["len"], None, MU0, EPS0, x["pe"], x["ge"], 1.0, x["spread"], 50.0,
                     opts=sweep_opts(solver=solver, scheme="extract", batch=batch, graphs=graphs, nfreq_hint=nfreq),
                     rule_order=-7,
                     ctx=ctx)


def features(d: PatchDesign, freqs):
    """Normalised network inputs [n x 5] (float32)."""
    f = np.asarray(freqs, dtype=np.float64).reshape(-1)
    X = np.empty((f.size, 5), dtype=np.float32)
    X[:, 0] = (d.W - 35e-3) / 10e-3
    X[:, 1] = (d.L - 30e-3) / 10e-3
    X[:, 2] = (d.h - 2e-3) / 1.2e-3
    X[:, 3] = d.feed / (d.L / 3.0)
    X[:, 4] = (f / d.f0 - 1.0) / BAND
    return X


def zin_to_target(Zin):
    Zin = np.asarray(Zin, dtype=np.complex128).reshape(-1)
    a = np.abs(Zin)
    ph = Zin / np.where(a > 0, a, 1.0)
    return np.stack([np.log(np.maximum(a, 1e-300) / Z_SCALE), ph.real, ph.imag], axis=1).astype(np.float32)


def target_to_zin(T):
    T = np.asarray(T, dtype=np.float64)
    u = T[:, 1] + 1j * T[:, 2]
    n = np.abs(u)
    return Z_SCALE * np.exp(T[:, 0]) * u / np.where(n > 0, n, 1.0)


def s11(Zin, Z0=50.0):
    return (Zin - Z0) / (Zin + Z0)


# ---------------------------------------------------------------------------
# The network
# ---------------------------------------------------------------------------
class Surrogate:
    """The MLP of csrc/surrogate.cu (BF16 weights, FP32 accumulate)."""

    def __init__(self, n_in=5, n_hidden=256, n_layers=4, n_out=N_OUT, seed=1):
        cfg = nat.EfieMlpConfig(n_in, n_hidden, n_layers, n_out, seed)
        h = C.c_void_p()
        nat.check(nat.lib().efie_mlp_create(nat.context(), C.byref(cfg), C.byref(h)))
        self._h = h
        self.cfg = dict(n_in=n_in, n_hidden=n_hidden, n_layers=n_layers, n_out=n_out)
        self.shapes = [(n_in if l == 0 else n_hidden, n_out if l == n_layers else n_hidden)
                       for l in range(n_layers + 1)]
        self.n_params = int(nat.lib().efie_mlp_num_params(h))
        nat.register_plan(self)

    def get_params(self):
        p = np.zeros(self.n_params, dtype=np.float32)
        nat.check(nat.lib().efie_mlp_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.n_params
        nat.check(nat.lib().efie_mlp_set_params(self._h, p.ctypes.data))

    def forward(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros((X.shape[0], self.cfg["n_out"]), dtype=np.float32)
        nat.check(nat.lib().efie_mlp_forward(self._h, X.ctypes.data, X.shape[0], Y.ctypes.data))
        return Y

    def loss_grad(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_double()
        nat.check(nat.lib().efie_mlp_loss_grad(self._h, X.ctypes.data, T.ctypes.data, X.shape[0], C.byref(loss),
                                               g.ctypes.data))
        return loss.value, g

    def train(self, X, T, epochs=100, batch=1024, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0,
              seed=1):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        o = nat.EfieAdamOpts(lr, beta1, beta2, eps, weight_decay, batch, epochs, seed)
        hist = np.zeros(max(1, epochs), dtype=np.float64)
        nat.check(nat.lib().efie_mlp_train(self._h, X.ctypes.data, T.ctypes.data, X.shape[0], C.byref(o),
                                           hist.ctypes.data))
        return hist[:epochs]

    def predict_zin(self, d: PatchDesign, freqs):
        return target_to_zin(self.forward(features(d, freqs)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            nat.lib().efie_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Design families: several designs in flight at once
# ---------------------------------------------------------------------------
_worker_ctx = {}   # (device, worker) -> context of a sweep_family worker, kept for later calls


def _worker_context(device, w):
    key = (device, w)
    if key not in _worker_ctx:
        if not _worker_ctx:
            import atexit
            atexit.register(_release_worker_contexts)
        _worker_ctx[key] = nat.new_context(device)
    return _worker_ctx[key]


def _release_worker_contexts():
    for h in _worker_ctx.values():
        nat.destroy_context(h)
    _worker_ctx.clear()


def sweep_family(designs, nfreq, workers=2, device=0, solver="mixed", streams=None, times=None):
    """Zin over each design's band (``d.band(nfreq)``) for a family of
    designs of uneven Ne, ``workers`` designs in flight at once.

    Each worker is a host thread with a library context of its own (its own
    CUDA stream -- ``streams[w]`` when given, a ``cudaStream_t`` --, solver
    handle and look-ahead streams; the contexts are kept for later calls and
    released at exit): it meshes its next design on the GPU,
    creates the plan (extraction scheme), sweeps and releases it, while the
    other workers' designs run on their streams.  The latency-bound phases of
    one design (the LU's panel chain, GMRES's stop-flag polls, plan set-up on
    the host) then overlap the bulk kernels of the others.  Every design is
    solved exactly as design_plan(d).run(d.band(nfreq)) alone (the sweeps
    share nothing).  The factorizations launch eagerly instead of replaying
    a captured graph: a stream capture in one thread would be invalidated by
    the device-wide synchronisation that another thread's plan release
    performs.  Returns [(Ne, Zin)] in the order of ``designs``; a failure in
    any worker is raised after all workers have stopped.  ``times`` (a list,
    optional) receives one (mesh + plan set-up seconds, sweep seconds) pair
    per design, host wall clock in its worker thread."""
    import time
    import queue
    import threading
    out = [None] * len(designs)
    todo = queue.Queue()
    for i in range(len(designs)):
        todo.put(i)
    errors = []

    ctxs = [_worker_context(device, w) for w in range(max(1, workers))]   # created in this thread

    def work(w):
        ctx = ctxs[w]
        try:
            nat.check(nat.lib().efie_ctx_set_stream(ctx, streams[w] if streams is not None else None))
            while not errors:
                try:
                    i = todo.get_nowait()
                except queue.Empty:
                    return
                d = designs[i]
                t0 = time.perf_counter()
                plan = design_plan(d, solver=solver, ctx=ctx, graphs=False, nfreq=nfreq)
                t1 = time.perf_counter()
                try:
                    Zin, _ = plan.run(d.band(nfreq))
                    out[i] = (plan.Ne, Zin)
                    if times is not None:
                        times.append((t1 - t0, time.perf_counter() - t1))
                finally:
                    plan.close()
        except Exception as e:  # noqa: BLE001 -- re-raised below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(w,)) for w in range(max(1, workers))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return out


# ---------------------------------------------------------------------------
# Training data from the solver
# ---------------------------------------------------------------------------
def generate_samples(designs, n_freq, seed=0, solver="mixed"):
    """Zin of every design at n_freq random frequencies of its band: X, T, and
    the number of solved points."""
    rng = np.random.default_rng(seed)
    Xs, Ts = [], []
    for d in designs:
        fr = np.sort(d.f0 * (1.0 + BAND * rng.uniform(-1.0, 1.0, n_freq)))
        plan = design_plan(d, solver=solver)
        Zin, _ = plan.run(fr)
        plan.close()
        Xs.append(features(d, fr))
        Ts.append(zin_to_target(Zin))
    return np.concatenate(Xs), np.concatenate(Ts)


# ---------------------------------------------------------------------------
# Sweeps
# ---------------------------------------------------------------------------
def _refine_min(f, y):
    """Sub-grid minimum of sampled y(f) by a parabola through the smallest
    sample and its neighbours."""
    i = int(np.argmin(y))
    if 0 < i < len(f) - 1:
        y0, y1, y2 = y[i - 1], y[i], y[i + 1]
        den = y0 - 2 * y1 + y2
        if den > 0:
            t = 0.5 * (y0 - y2) / den
            return float(f[i] + t * (f[i + 1] - f[i]))
    return float(f[i])


def dense_sweep(d: PatchDesign, n=201, plan=None):
    """The plain sweep: n uniformly spaced solves over the design's band."""
    own = plan is None
    plan = plan or design_plan(d)
    fr = d.band(n)
    Zin, S = plan.run(fr)
    if own:
        plan.close()
    return dict(freqs=fr, Zin=Zin, S11=S, f_min=_refine_min(fr, np.abs(S)), solves=n)


def _interp_correction(fs, dz, fq):
    """Smooth interpolant of complex samples dz at the frequencies fs,
    evaluated at fq: a not-a-knot cubic spline (a polynomial through the
    points when there are fewer than four), held constant outside [min fs,
    max fs]."""
    from scipy.interpolate import CubicSpline

    o = np.argsort(fs)
    fs, dz = np.asarray(fs, np.float64)[o], np.asarray(dz, np.complex128)[o]
    fq = np.clip(np.asarray(fq, np.float64), fs[0], fs[-1])
    if fs.size == 1:
        return np.full(fq.shape, dz[0])
    if fs.size < 4:
        c = np.polyfit(fs - fs[0], dz, fs.size - 1)
        return np.polyval(c, fq - fs[0])
    return CubicSpline(fs, dz.real)(fq) + 1j * CubicSpline(fs, dz.imag)(fq)


def adaptive_sweep(d: PatchDesign, net: Surrogate, plan=None, n_points=8, tol=1e-3, max_rounds=4, n_dense=201,
                   span=0.04):
    """Locate the |S11| minimum of a design with few EFIE solves.

    Round 1 solves n_points around the surrogate's predicted minimum (spread
    over +-span * f0); each later round solves n_points around the current
    estimate with half the previous spread.  Between solved points the curve
    is the surrogate plus an interpolant of its error at the solved points.
    A round converges when the minimum is bracketed by solved points (or sits
    at a band edge a solved point reaches) and either the corrected surrogate
    predicted the round's new solves within ``tol`` (relative |dZin|) or the
    minimum moved by less than 0.1 dense-grid step since the previous round.
    Other dips of the raw surrogate that come within its observed |S11| error
    of the found minimum are then solved too (n_points / 2 each), so that a
    secondary minimum is not taken for the global one.  Without convergence
    after max_rounds the sweep falls back to the dense plain sweep of n_dense
    points (the full solve).
    """
    own = plan is None
    plan = plan or design_plan(d)
    fq = d.band(4 * (n_dense - 1) + 1)
    step = (fq[-1] - fq[0]) / (n_dense - 1)
    zs = net.predict_zin(d, fq)
    f_est = _refine_min(fq, np.abs(s11(zs)))
    lo, hi = fq[0], fq[-1]
    fs = np.zeros(0)
    zsol = np.zeros(0, dtype=complex)
    sp = span * d.f0
    rounds = 0
    converged = False
    err_pred = np.inf

    def corrected(fs, zsol):
        return zs + _interp_correction(fs, zsol - net.predict_zin(d, fs), fq)

    def solve(new):
        nonlocal fs, zsol
        new = np.setdiff1d(np.unique(np.clip(new, lo, hi)), fs)
        if new.size == 0:
            return new, np.zeros(0, complex)
        zn, _ = plan.run(new)
        fs = np.concatenate([fs, new])
        zsol = np.concatenate([zsol, zn])
        return new, zn

    while rounds < max_rounds:
        rounds += 1
        cand = f_est + sp * np.linspace(-1.0, 1.0, n_points)
        pred_all = corrected(fs, zsol) if fs.size else zs
        new, zn = solve(cand)
        if new.size == 0:
            break
        # the corrected surrogate's prediction of the new points, before solving them
        pred = np.interp(new, fq, pred_all.real) + 1j * np.interp(new, fq, pred_all.imag)
        err_pred = float(np.max(np.abs(pred - zn) / np.abs(zn)))
        f_prev = f_est
        f_est = _refine_min(fq, np.abs(s11(corrected(fs, zsol))))
        tol_f = 1e-9 * d.f0
        inside = (fs.min() < f_est < fs.max()) or (f_est <= lo + tol_f and fs.min() <= lo + tol_f) or \
                 (f_est >= hi - tol_f and fs.max() >= hi - tol_f)
        stable = rounds > 1 and abs(f_est - f_prev) <= 0.1 * step
        if inside and (err_pred <= tol or stable):
            converged = True
            break
        sp *= 0.5
    if converged:
        # other dips of the surrogate within its observed error of the found minimum
        s_raw = np.abs(s11(zs))
        s_at = np.abs(s11(net.predict_zin(d, fs)))
        delta = 3.0 * float(np.max(np.abs(s_at - np.abs(s11(zsol)))))
        best = float(np.min(np.abs(s11(corrected(fs, zsol)))))
        i = np.arange(1, fq.size - 1)
        dips = i[(s_raw[i] <= s_raw[i - 1]) & (s_raw[i] <= s_raw[i + 1])]
        dips = [fq[k] for k in dips if s_raw[k] <= best + delta and not (fs.min() <= fq[k] <= fs.max())]
        for c in sorted(dips, key=lambda f: np.interp(f, fq, s_raw))[:3]:
            solve(c + 0.5 * span * d.f0 * np.linspace(-1.0, 1.0, max(2, n_points // 2)))
        f_est = _refine_min(fq, np.abs(s11(corrected(fs, zsol))))
    result = dict(f_min=f_est, solves=int(fs.size), rounds=rounds, converged=converged, err_pred=err_pred,
                  fallback=False, freqs=fs, Zin=zsol)
    if not converged:
        dn = dense_sweep(d, n_dense, plan)
        result.update(f_min=dn["f_min"], solves=int(fs.size) + n_dense, fallback=True)
    if own:
        plan.close()
    return result


def uniform_sweep_estimate(d: PatchDesign, n, plan=None, n_fine=801):
    """The method without the network at the same budget: n uniform solves
    over the band and a cubic interpolant of Zin between them."""
    own = plan is None
    plan = plan or design_plan(d)
    fr = d.band(n)
    Zin, _ = plan.run(fr)
    if own:
        plan.close()
    fq = d.band(n_fine)
    zi = _interp_correction(fr, Zin, fq)
    return dict(f_min=_refine_min(fq, np.abs(s11(zi))), solves=n)
