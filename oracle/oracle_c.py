"""ctypes binding of the C oracle (``oracle/efie_oracle.c``).

TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline); see the header of
``efie_oracle.c``.  Builds ``oracle/liboracle.so`` on first use if missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build(force=False):
    src = os.path.join(HERE, "efie_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-o", LIB, src, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def assemble_z(rwg, prepack, k, omega, mu, eps, col0=0, col1=None, nthreads=0):
    """Z (complex128, Ne x Ne, Fortran order) of CPU_FAST for columns [col0, col1)."""
    Ne = int(rwg["Ne"])
    col1 = Ne if col1 is None else col1
    Nq, _, Nt = prepack["r_reg"].shape
    Nq2, _, NsS, _ = prepack["self_r"].shape
    NsN = prepack["near_r"].shape[2]
    i32 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1, order="F"))
    f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, order="F"))
    arrs = dict(pt=i32(rwg["plusTri"]), mt=i32(rwg["minusTri"]), ps=i32(rwg["plusSign"]),
                ms=i32(rwg["minusSign"]), rp=f64(rwg["rp"]), rm=f64(rwg["rm"]), Ap=f64(rwg["Ap"]),
                Am=f64(rwg["Am"]), ln=f64(rwg["len"]), rr=f64(prepack["r_reg"]), wr=f64(prepack["w_reg"]),
                nm=np.ascontiguousarray(np.asarray(prepack["nearMat"], dtype=np.uint8).reshape(-1, order="F")),
                sr=f64(prepack["self_r"]), sw=f64(prepack["self_w"]), sa=f64(prepack["self_a"]),
                nr=f64(prepack["near_r"]), nw=f64(prepack["near_w"]), aq=f64(prepack["aeqTri"]))
    Z = np.zeros((Ne, Ne), dtype=np.complex128, order="F")
    L = lib()
    L.oracle_assemble_z.restype = C.c_int
    k = complex(k)
    eps = complex(eps)
    rc = L.oracle_assemble_z(
        C.c_int(Ne), C.c_int(Nt), C.c_int(Nq), C.c_int(Nq2), C.c_int(NsS), C.c_int(NsN),
        _p(arrs["pt"], C.c_int32), _p(arrs["mt"], C.c_int32), _p(arrs["ps"], C.c_int32), _p(arrs["ms"], C.c_int32),
        _p(arrs["rp"], C.c_double), _p(arrs["rm"], C.c_double), _p(arrs["Ap"], C.c_double),
        _p(arrs["Am"], C.c_double), _p(arrs["ln"], C.c_double),
        _p(arrs["rr"], C.c_double), _p(arrs["wr"], C.c_double), _p(arrs["nm"], C.c_uint8),
        _p(arrs["sr"], C.c_double), _p(arrs["sw"], C.c_double), _p(arrs["sa"], C.c_double),
        _p(arrs["nr"], C.c_double), _p(arrs["nw"], C.c_double), _p(arrs["aq"], C.c_double),
        C.c_double(prepack["near_alpha"]),
        C.c_double(k.real), C.c_double(k.imag), C.c_double(omega), C.c_double(mu),
        C.c_double(eps.real), C.c_double(eps.imag), C.c_int(col0), C.c_int(col1),
        Z.ctypes.data_as(C.POINTER(C.c_double)), C.c_int(nthreads))
    if rc != 0:
        raise RuntimeError("oracle_assemble_z failed: %d" % rc)
    return Z


def assemble_centroid(V, F, rwg, self_alpha, k, omega, mu, eps, nthreads=0):
    """Z of the centroid kernel (gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:49-106)."""
    Ne = int(rwg["Ne"])
    Vf = np.ascontiguousarray(np.asarray(V, dtype=np.float64).reshape(-1, order="F"))
    Ff = np.ascontiguousarray(np.asarray(F, dtype=np.int32).reshape(-1, order="F"))
    i32 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1, order="F"))
    f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, order="F"))
    pt, mt, ps, ms = (i32(rwg[x]) for x in ("plusTri", "minusTri", "plusSign", "minusSign"))
    rp, rm, Ap, Am, ln = (f64(rwg[x]) for x in ("rp", "rm", "Ap", "Am", "len"))
    Z = np.zeros((Ne, Ne), dtype=np.complex128, order="F")
    k = complex(k)
    eps = complex(eps)
    L = lib()
    rc = L.oracle_assemble_centroid(
        C.c_int(np.asarray(V).shape[0]), C.c_int(np.asarray(F).shape[0]), C.c_int(Ne),
        _p(Vf, C.c_double), _p(Ff, C.c_int32), _p(pt, C.c_int32), _p(mt, C.c_int32),
        _p(ps, C.c_int32), _p(ms, C.c_int32), _p(rp, C.c_double), _p(rm, C.c_double),
        _p(Ap, C.c_double), _p(Am, C.c_double), _p(ln, C.c_double),
        C.c_double(self_alpha), C.c_double(k.real), C.c_double(k.imag), C.c_double(omega),
        C.c_double(mu), C.c_double(eps.real), C.c_double(eps.imag),
        Z.ctypes.data_as(C.POINTER(C.c_double)), C.c_int(nthreads))
    if rc != 0:
        raise RuntimeError("oracle_assemble_centroid failed: %d" % rc)
    return Z


def potential_integrals(a, r):
    """Analytic I0, J of the C oracle (oracle_potential_integrals)."""
    L = lib()
    aa = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(3, 3))
    rr = np.ascontiguousarray(np.asarray(r, dtype=np.float64).reshape(3))
    I0 = C.c_double()
    J = np.zeros(3)
    L.oracle_potential_integrals(_p(aa, C.c_double), _p(rr, C.c_double), C.byref(I0), _p(J, C.c_double))
    return I0.value, J


def assemble_z_extract(V, F, rwg, k, omega, mu, eps, rule=-7, col0=0, col1=None, nthreads=0):
    """Z of the extraction scheme (Dunavant 7-point rule by default)."""
    import efie_oracle as eo
    qp, qw = eo.tri_quad_rule(rule)
    Ne = int(rwg["Ne"])
    col1 = Ne if col1 is None else col1
    Vf = np.ascontiguousarray(np.asarray(V, dtype=np.float64).reshape(-1, order="F"))
    Ff = np.ascontiguousarray(np.asarray(F, dtype=np.int32).reshape(-1, order="F"))
    i32 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1, order="F"))
    f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, order="F"))
    pt, mt, ps, ms = (i32(rwg[x]) for x in ("plusTri", "minusTri", "plusSign", "minusSign"))
    rp, rm, Ap, Am, ln = (f64(rwg[x]) for x in ("rp", "rm", "Ap", "Am", "len"))
    qu, qv, qww = (np.ascontiguousarray(x, dtype=np.float64) for x in (qp[:, 0], qp[:, 1], qw))
    Z = np.zeros((Ne, Ne), dtype=np.complex128, order="F")
    k = complex(k)
    eps = complex(eps)
    L = lib()
    rc = L.oracle_assemble_z_extract(
        C.c_int(np.asarray(V).shape[0]), C.c_int(np.asarray(F).shape[0]), C.c_int(Ne), _p(Vf, C.c_double),
        _p(Ff, C.c_int32), _p(pt, C.c_int32), _p(mt, C.c_int32), _p(ps, C.c_int32), _p(ms, C.c_int32),
        _p(rp, C.c_double), _p(rm, C.c_double), _p(Ap, C.c_double), _p(Am, C.c_double), _p(ln, C.c_double),
        C.c_int(len(qw)), _p(qu, C.c_double), _p(qv, C.c_double), _p(qww, C.c_double),
        C.c_double(k.real), C.c_double(k.imag), C.c_double(omega), C.c_double(mu), C.c_double(eps.real),
        C.c_double(eps.imag), C.c_int(col0), C.c_int(col1), Z.ctypes.data_as(C.POINTER(C.c_double)),
        C.c_int(nthreads))
    if rc != 0:
        raise RuntimeError("oracle_assemble_z_extract failed: %d" % rc)
    return Z
