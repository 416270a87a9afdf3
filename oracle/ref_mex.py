"""Calls the reference's own MEX functions, compiled unmodified for sm_100a
against the fake mex shim (``oracle/Makefile`` -> ``oracle/_ref/*.so``).

TEST INFRASTRUCTURE ONLY: used by the GPU parity tests to pin the oracle and
by bench.py to time the reference GPU code; never by the product.
Needs a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
MX_DOUBLE, MX_INT32, MX_UINT8 = 6, 12, 9


class RefError(RuntimeError):
    def __init__(self, ident, msg):
        super().__init__("%s: %s" % (ident, msg))
        self.identifier = ident


class RefMex:
    def __init__(self, name):
        path = os.path.join(REF_DIR, name + ".so")
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (build with: make -C oracle)")
        L = C.CDLL(path)
        L.fm_numeric.restype = C.c_void_p
        L.fm_numeric.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_size_t), C.c_void_p, C.c_void_p]
        L.fm_struct.restype = C.c_void_p
        L.fm_struct.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_void_p)]
        L.fm_destroy.argtypes = [C.c_void_p]
        L.fm_numel.restype = C.c_size_t
        L.fm_numel.argtypes = [C.c_void_p]
        L.fm_read.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.fm_call.restype = C.c_int
        L.fm_call.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p),
                              C.c_char_p, C.c_char_p, C.c_int]
        self.L = L

    def _mx(self, a):
        if isinstance(a, dict):
            names = list(a.keys())
            vals = [self._mx(a[k]) for k in names]
            arr_n = (C.c_char_p * len(names))(*[n.encode() for n in names])
            arr_v = (C.c_void_p * len(vals))(*vals)
            return self.L.fm_struct(len(names), arr_n, arr_v)
        a = np.asarray(a)
        if a.dtype == np.int32:
            cls = MX_INT32
        elif a.dtype == np.uint8:
            cls = MX_UINT8
        else:
            cls = MX_DOUBLE
        dims = list(a.shape)
        while len(dims) < 2:
            dims.append(1)
        dims_c = (C.c_size_t * len(dims))(*dims)
        if np.iscomplexobj(a):
            re = np.ascontiguousarray(a.real.astype(np.float64).reshape(-1, order="F"))
            im = np.ascontiguousarray(a.imag.astype(np.float64).reshape(-1, order="F"))
            return self.L.fm_numeric(cls, len(dims), dims_c, re.ctypes.data, im.ctypes.data)
        if cls == MX_DOUBLE:
            a = a.astype(np.float64)
        re = np.ascontiguousarray(a.reshape(-1, order="F"))
        return self.L.fm_numeric(cls, len(dims), dims_c, re.ctypes.data, None)

    def call(self, nlhs, *args):
        prhs = [self._mx(a) for a in args]
        pr = (C.c_void_p * max(len(prhs), 1))(*prhs)
        pl = (C.c_void_p * max(nlhs, 1))()
        eid = C.create_string_buffer(512)
        emsg = C.create_string_buffer(512)
        try:
            rc = self.L.fm_call(nlhs, pl, len(prhs), pr, eid, emsg, 512)
            if rc != 0:
                raise RefError(eid.value.decode(), emsg.value.decode())
            outs = []
            for i in range(nlhs):
                n = self.L.fm_numel(pl[i])
                re = np.zeros(n)
                im = np.zeros(n)
                self.L.fm_read(pl[i], re.ctypes.data, im.ctypes.data)
                outs.append(re + 1j * im)
                self.L.fm_destroy(pl[i])
            return outs
        finally:
            for p in prhs:
                self.L.fm_destroy(p)


def ggassemble(prob, k, omega, mu, eps):
    """Reference ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST -> (Z [Ne x Ne], Vrhs [Ne])."""
    r = prob["rwg"]
    exc = np.array([prob["patchEdge"], prob["groundEdge"], prob["design"].V0, prob["spread"]], dtype=np.float64)
    Z, V = RefMex("ggassemble_ref").call(
        2, prob["V"], prob["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"],
        r["rp"], r["rm"], r["Ap"], r["Am"], r["len"], prob["prepack"], complex(k), omega, mu, complex(eps), exc)
    Ne = r["Ne"]
    return Z.reshape(Ne, Ne, order="F"), V


def gassemble(prob, k, omega, mu, eps, self_alpha=0.2):
    r = prob["rwg"]
    exc = np.array([prob["patchEdge"], prob["groundEdge"], prob["design"].V0, prob["spread"], self_alpha])
    Z, V = RefMex("gassemble_ref").call(
        2, prob["V"], prob["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"],
        r["rp"], r["rm"], r["Ap"], r["Am"], r["len"], complex(k), omega, mu, complex(eps), exc)
    Ne = r["Ne"]
    return Z.reshape(Ne, Ne, order="F"), V


def patch_sweep_fastquad(prob, freqs):
    r = prob["rwg"]
    d = prob["design"]
    Zin, S11 = RefMex("patch_sweep_fastquad_ref").call(
        2, prob["V"], prob["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"],
        r["rp"], r["rm"], r["Ap"], r["Am"], r["len"], prob["prepack"], np.asarray(freqs, np.float64),
        d.mu, complex(d.eps), float(prob["patchEdge"]), float(prob["groundEdge"]), d.V0, prob["spread"], d.Z0)
    return Zin, S11


def patch_sweep_cuda(prob, freqs):
    r = prob["rwg"]
    d = prob["design"]
    Zin, S11 = RefMex("patch_sweep_cuda_ref").call(
        2, prob["V"], prob["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"],
        r["rp"], r["rm"], r["Ap"], r["Am"], r["len"], np.asarray(freqs, np.float64), d.mu, complex(d.eps),
        np.int32(prob["patchEdge"]), np.int32(prob["groundEdge"]), d.V0, prob["spread"], d.Z0)
    return Zin, S11
