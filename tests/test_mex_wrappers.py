"""The C MEX wrappers (matlab-cuda-efief-vs-cpu_b200/mex/*.c) compiled against
the fake mex shim: on CPU they must reject bad arguments with the reference's
error identifiers; on a GPU they must reproduce the Python mirror."""
import os
import subprocess

import numpy as np
import pytest

import efie_oracle as eo
from conftest import ROOT, small_design

MEXDIR = os.path.join(ROOT, "matlab-cuda-efief-vs-cpu_b200", "mex")
LIBDIR = os.path.join(ROOT, "matlab-cuda-efief-vs-cpu_b200")
SHIM = os.path.join(ROOT, "oracle", "fake_mex")
WRAPPERS = ["ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST", "gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST",
            "patch_sweep_fastquad_cuda", "patch_sweep_cuda"]


@pytest.fixture(scope="session")
def mexlibs(tmp_path_factory):
    out = tmp_path_factory.mktemp("mex")
    shim_o = os.path.join(out, "fake_mex.o")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-fPIC", "-I", SHIM, "-c",
                           os.path.join(SHIM, "fake_mex.cpp"), "-o", shim_o])
    libs = {}
    for w in WRAPPERS:
        o = os.path.join(out, w + ".o")
        subprocess.check_call(["gcc", "-std=c99", "-O2", "-fPIC", "-Wall", "-Werror", "-I", SHIM, "-I",
                               os.path.join(ROOT, "include"), "-c", os.path.join(MEXDIR, w + ".c"), "-o", o])
        so = os.path.join(out, w + ".so")
        subprocess.check_call(["g++", "-shared", "-o", so, o, shim_o, "-L", LIBDIR, "-lefie_b200",
                               "-Wl,-rpath," + LIBDIR])
        libs[w] = so
    return libs


def _call(libs, name, nlhs, *args):
    import ref_mex
    m = ref_mex.RefMex.__new__(ref_mex.RefMex)
    ref_mex.RefMex.__init__.__globals__  # noqa: B018 (module import side effect)
    import ctypes as C
    L = C.CDLL(libs[name])
    for fn, res, at in (("fm_numeric", C.c_void_p, [C.c_int, C.c_int, C.POINTER(C.c_size_t), C.c_void_p, C.c_void_p]),
                        ("fm_struct", C.c_void_p, [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_void_p)]),
                        ("fm_destroy", None, [C.c_void_p]), ("fm_numel", C.c_size_t, [C.c_void_p]),
                        ("fm_read", None, [C.c_void_p, C.c_void_p, C.c_void_p]),
                        ("fm_call", C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p),
                                              C.c_char_p, C.c_char_p, C.c_int])):
        getattr(L, fn).restype = res
        getattr(L, fn).argtypes = at
    m.L = L
    return m.call(nlhs, *args)


def _base(p):
    r = p["rwg"]
    return [p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
            r["Ap"], r["Am"], r["len"]]


def _err(libs, name, nlhs, *args):
    import ref_mex
    with pytest.raises(ref_mex.RefError) as e:
        _call(libs, name, nlhs, *args)
    return e.value.identifier


def test_wrappers_reject_bad_arguments(mexlibs, small_problem):
    p = small_problem
    d = p["design"]
    base = _base(p)
    exc4 = np.array([p["patchEdge"], p["groundEdge"], 1.0, p["spread"]])
    gg = "ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST"
    args = base + [p["prepack"], 2.0 + 0j, 1e10, d.mu, complex(d.eps), exc4]
    assert _err(mexlibs, gg, 2, *args[:17]) == "mex:args"
    assert _err(mexlibs, gg, 1, *args) == "mex:args"
    b = list(args); b[1] = p["F"].astype(np.float64); assert _err(mexlibs, gg, 2, *b) == "mex:F"
    b = list(args); b[17] = np.array([0.0, 1, 1, 1]); assert _err(mexlibs, gg, 2, *b) == "mex:port"
    b = list(args); pr = dict(p["prepack"]); del pr["near_w"]; b[12] = pr
    assert _err(mexlibs, gg, 2, *b) == "mex:prepack"
    b = list(args); pr = dict(p["prepack"]); pr["nearMat"] = pr["nearMat"].astype(np.float64); b[12] = pr
    assert _err(mexlibs, gg, 2, *b) == "mex:nearMat"
    g = "gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST"
    exc5 = np.array([p["patchEdge"], p["groundEdge"], 1.0, p["spread"], 0.2])
    args = base + [2.0 + 0j, 1e10, d.mu, complex(d.eps), exc5]
    b = list(args); b[4] = p["rwg"]["minusTri"].astype(np.float64); assert _err(mexlibs, g, 2, *b) == "mex:minusTri"
    b = list(args); b[16] = exc5[:4]; assert _err(mexlibs, g, 2, *b) == "mex:exc"
    s = "patch_sweep_cuda"
    fr = np.array([2e9, 2.5e9])
    args = base + [fr, d.mu, complex(d.eps), np.int32(p["patchEdge"]), np.int32(p["groundEdge"]), 1.0, p["spread"],
                   50.0]
    b = list(args); b[2] = p["rwg"]["edge"].astype(np.float64); assert _err(mexlibs, s, 2, *b) == "mex:edge"
    b = list(args); b[15] = np.int32(0); assert _err(mexlibs, s, 2, *b) == "mex:port"


@pytest.mark.gpu
def test_wrappers_match_python_mirror(mexlibs, small_problem):
    import importlib
    m = importlib.import_module("matlab-cuda-efief-vs-cpu_b200")
    p = small_problem
    d = p["design"]
    base = _base(p)
    omega, k, _, _ = eo.physics(2.4e9, d.mu, d.eps)
    exc4 = np.array([p["patchEdge"], p["groundEdge"], 1.0, p["spread"]])
    Z, V = _call(mexlibs, "ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST", 2, *base, p["prepack"], complex(k), omega, d.mu,
                 complex(d.eps), exc4)
    Zp, Vp = m.ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(*base, p["prepack"], k, omega, d.mu, d.eps, exc4)
    Ne = p["rwg"]["Ne"]
    assert np.array_equal(Z.reshape(Ne, Ne, order="F"), Zp) and np.array_equal(V, Vp)
    fr = d.freqs
    Zin, S11 = _call(mexlibs, "patch_sweep_fastquad_cuda", 2, *base, p["prepack"], fr, d.mu, complex(d.eps),
                     float(p["patchEdge"]), float(p["groundEdge"]), 1.0, p["spread"], 50.0)
    Zi2, S2 = m.patch_sweep_fastquad_cuda(*base, p["prepack"], fr, d.mu, d.eps, p["patchEdge"], p["groundEdge"], 1.0,
                                          p["spread"], 50.0)
    assert np.abs(Zin - Zi2).max() <= 1e-9 * np.abs(Zi2).max()
