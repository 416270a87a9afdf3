"""CPU tests of the C ABI boundary: the library loads, exports every symbol
that include/efie_b200.h declares, and the host mirror rejects bad arguments
with the reference's error identifiers before touching a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import efie_oracle as eo
from conftest import pkg, small_design

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "efie_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(efie_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    m = pkg()
    L = m.lib()
    syms = _declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s


def test_binding_covers_header():
    from importlib import import_module
    nat = import_module("matlab-cuda-efief-vs-cpu_b200._native")
    assert set(_declared_symbols()) == set(nat.SIGNATURES)


def test_status_ids():
    m = pkg()
    L = m.lib()
    assert L.efie_status_id(6) == b"mex:port"
    assert L.efie_status_id(21) == b"cuda:rt"
    assert L.efie_status_id(22) == b"cuda:cusolver"


def _args(p, k=2.0 + 0j, omega=1e10):
    r = p["rwg"]
    d = p["design"]
    exc = np.array([p["patchEdge"], p["groundEdge"], d.V0, p["spread"]], dtype=np.float64)
    return [p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"],
            r["rm"], r["Ap"], r["Am"], r["len"], p["prepack"], k, omega, d.mu, d.eps, exc]


def _ident(fn, *a, **kw):
    with pytest.raises(pkg().MexError) as e:
        fn(*a, **kw)
    return e.value.identifier


def test_ggassemble_argument_errors(small_problem):
    m = pkg()
    f = m.ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST
    a = _args(small_problem)
    assert _ident(f, *a[:17]) == "mex:args"
    assert _ident(f, *a, nargout=1) == "mex:args"
    b = list(a); b[0] = a[0][:, :2].copy(); assert _ident(f, *b) == "mex:V"
    b = list(a); b[1] = a[1].astype(np.float64); assert _ident(f, *b) == "mex:F"
    b = list(a); b[2] = a[2].astype(np.int64); assert _ident(f, *b) == "mex:E"
    b = list(a); b[12] = None; assert _ident(f, *b) == "mex:prepack"
    b = list(a); b[17] = a[17][:3].copy(); assert _ident(f, *b) == "mex:exc"
    b = list(a); e = a[17].copy(); e[0] = 0; b[17] = e; assert _ident(f, *b) == "mex:port"
    b = list(a); e = a[17].copy(); e[1] = small_problem["rwg"]["Ne"] + 1; b[17] = e; assert _ident(f, *b) == "mex:port"
    for fld, ident in (("r_reg", "mex:prepack"), ("nearMat", "mex:prepack")):
        b = list(a); pr = dict(a[12]); del pr[fld]; b[12] = pr; assert _ident(f, *b) == ident
    b = list(a); pr = dict(a[12]); pr["nearMat"] = pr["nearMat"].astype(np.float64); b[12] = pr
    assert _ident(f, *b) == "mex:nearMat"
    b = list(a); pr = dict(a[12]); pr["aeqTri"] = pr["aeqTri"][:-1]; b[12] = pr
    assert _ident(f, *b) == "mex:aeqTri"
    b = list(a); pr = dict(a[12]); pr["self_r"] = pr["self_r"][:, :2]; b[12] = pr
    assert _ident(f, *b) == "mex:self_r"


def test_gassemble_and_sweep_argument_errors(small_problem):
    m = pkg()
    p = small_problem
    r = p["rwg"]
    d = p["design"]
    base = [p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
            r["Ap"], r["Am"], r["len"]]
    g = m.gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST
    exc5 = np.array([p["patchEdge"], p["groundEdge"], 1.0, p["spread"], 0.2])
    args = base + [2.0, 1e10, d.mu, d.eps, exc5]
    b = list(args); b[3] = r["plusTri"].astype(np.float64); assert _ident(g, *b) == "mex:plusTri"
    b = list(args); b[7] = r["rp"][:, :2].copy(); assert _ident(g, *b) == "mex:rp"
    b = list(args); b[10] = r["Am"][:-1]; assert _ident(g, *b) == "mex:Am"
    b = list(args); b[16] = exc5[:4].copy(); assert _ident(g, *b) == "mex:exc"
    s = m.patch_sweep_fastquad_cuda
    fr = np.array([2e9, 2.5e9])
    sargs = base + [p["prepack"], fr, d.mu, d.eps, p["patchEdge"], p["groundEdge"], 1.0, p["spread"], 50.0]
    assert _ident(s, *sargs[:20]) == "mex:args"
    b = list(sargs); b[13] = fr.astype(np.float32); assert _ident(s, *b) == "mex:freqs"
    b = list(sargs); b[16] = 0; assert _ident(s, *b) == "mex:port"
    c = m.patch_sweep_cuda
    cargs = base + [fr, d.mu, d.eps, p["patchEdge"], p["groundEdge"], 1.0, p["spread"], 50.0]
    b = list(cargs); b[2] = r["edge"].astype(np.float64); assert _ident(c, *b) == "mex:edge"
    b = list(cargs); b[6] = r["minusSign"][:-1]; assert _ident(c, *b) == "mex:minusSign"
