"""Host-side mirror of the reference's MEX and MATLAB interface for the EFIE
hot path, calling the CUDA library only through its C ABI.

Function names, argument order, dtype/shape checks and error identifiers
follow the reference MEX functions:

* ``ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST``  (ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:542-657)
* ``gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST``   (gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:125-203)
* ``patch_sweep_fastquad_cuda``             (patch_sweep_fastquad_cuda.cu:461-580)
* ``patch_sweep_cuda``                      (patch_sweep_cuda.cu:172-225)
* ``assemble_ZV_EFIE_RWG_DIFF_GPU_FAST``    (assemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:277-378)

and the MATLAB producers of their inputs (make_patch_with_ground_mesh.m,
build_rwg_interior.m, pick_port_edge_by_point_and_layer.m,
efie_precompute.m + efie_precompute_pack.m).  Arrays are numpy arrays with
MATLAB semantics: index arrays int32 and 1-based, matrices column-major.
Errors raise ``MexError`` whose ``identifier`` is the reference's ID.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from ._native import MexError

__all__ = [
    "MexError", "ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST", "gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST",
    "patch_sweep_fastquad_cuda", "patch_sweep_cuda", "assemble_ZV_EFIE_RWG_DIFF_GPU_FAST",
    "make_patch_with_ground_mesh", "build_rwg_interior", "pick_port_edge_by_point_and_layer",
    "efie_precompute_pack", "efie_precompute_pack_gpu", "build_patch_design_gpu", "quad_rule_size", "SweepPlan",
    "sweep_opts",
]


# ---------------------------------------------------------------------------
# mxArray-like helpers
# ---------------------------------------------------------------------------
def _mx_dims(a):
    """MATLAB dimensions: at least 2, trailing singleton dimensions dropped."""
    s = list(np.shape(a))
    while len(s) > 2 and s[-1] == 1:
        s.pop()
    while len(s) < 2:
        s.append(1)
    return s


def _mx_M(a):
    return _mx_dims(a)[0]


def _mx_N(a):
    d = _mx_dims(a)
    return int(np.prod(d[1:]))


def _is(a, dt):
    return isinstance(a, np.ndarray) and a.dtype == dt


def _need(cond, ident, msg):
    if not cond:
        raise MexError(ident, msg)


def _scalar(a):
    a = np.asarray(a)
    return a.reshape(-1)[0].item() if a.size else 0.0


def _cscalar(a):
    v = complex(_scalar(a))
    return nat.c128(v.real, v.imag)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, order="F"))


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1, order="F"))


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class _Marshal:
    """Keeps the flattened copies alive while the C structs point at them."""

    def __init__(self):
        self.keep = []

    def f64(self, a):
        b = _f64(a)
        self.keep.append(b)
        return _ptr(b, C.c_double)

    def i32(self, a):
        b = _i32(a)
        self.keep.append(b)
        return _ptr(b, C.c_int32)

    def u8(self, a):
        b = np.ascontiguousarray(np.asarray(a, dtype=np.uint8).reshape(-1, order="F"))
        self.keep.append(b)
        return _ptr(b, C.c_uint8)

    def mesh(self, V, F, E, plusTri, minusTri, plusSign, minusSign, rp, rm, Ap, Am, length):
        Ne = _mx_M(E) if E is not None else np.size(plusTri)
        return nat.EfieMesh(
            _mx_M(V), _mx_M(F), Ne, self.f64(V), self.i32(F),
            self.i32(E) if E is not None else None,
            self.i32(plusTri), self.i32(minusTri), self.i32(plusSign), self.i32(minusSign),
            self.f64(rp), self.f64(rm), self.f64(Ap), self.f64(Am), self.f64(length))

    def prepack(self, pre, Nt, self_a_key="self_a", near_alpha=None):
        Nq = _mx_dims(pre["r_reg"])[0]
        sd = list(np.shape(pre["self_r"])) + [1, 1, 1, 1]
        Nq2, NsS = sd[0], sd[2]
        NsN = (list(np.shape(pre["near_r"])) + [1, 1, 1, 1])[2]
        na = _scalar(pre["near_alpha"]) if near_alpha is None else near_alpha
        sa = _scalar(pre["self_alpha"]) if "self_alpha" in pre else 0.0
        return nat.EfiePrepack(
            Nt, Nq, Nq2, NsS, NsN, self.f64(pre["r_reg"]), self.f64(pre["w_reg"]),
            self.u8(pre["nearMat"]), self.f64(pre["self_r"]), self.f64(pre["self_w"]),
            self.f64(pre[self_a_key]), self.f64(pre["near_r"]), self.f64(pre["near_w"]),
            self.f64(pre["aeqTri"]), float(na), float(sa))


def _check_VFE(V, F, E, e_id="mex:E", e_msg="E must be [Ne x 2] int32."):
    _need(_is(V, np.float64) and _mx_N(V) == 3, "mex:V", "V must be [Nv x 3] double.")
    _need(_is(F, np.int32) and _mx_N(F) == 3, "mex:F", "F must be [Nt x 3] int32.")
    _need(_is(E, np.int32) and _mx_N(E) == 2, e_id, e_msg)
    return _mx_M(V), _mx_M(F), _mx_M(E)


def _check_rwg_arrays(Ne, plusTri, minusTri, plusSign, minusSign, rp, rm, Ap, Am, length):
    # gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:181-191 / patch_sweep_cuda.cu:210-219
    for nm, a in (("plusTri", plusTri), ("minusTri", minusTri), ("plusSign", plusSign), ("minusSign", minusSign)):
        _need(_is(a, np.int32) and _mx_M(a) == Ne, "mex:" + nm, "%s must be int32 [Ne x 1]." % nm)
    for nm, a in (("rp", rp), ("rm", rm)):
        _need(_is(a, np.float64) and _mx_M(a) == Ne and _mx_N(a) == 3, "mex:" + nm,
              "%s must be [Ne x 3] double." % nm)
    for nm, a in (("Ap", Ap), ("Am", Am), ("len", length)):
        _need(_is(a, np.float64) and np.size(a) == Ne, "mex:" + nm, "%s must be [Ne x 1] double." % nm)


_PREPACK_FIELDS = ("r_reg", "w_reg", "nearMat", "self_r", "self_w", "self_a", "near_r", "near_w",
                   "aeqTri", "near_alpha")


def _get_field(pre, name, ident="mex:prepack", msg="Missing field in prepack."):
    _need(name in pre, ident, msg)
    return pre[name]


def _check_prepack_dims(pre, Nt):
    # ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:629-657
    r_reg = pre["r_reg"]
    _need(_is(r_reg, np.float64) and len(_mx_dims(r_reg)) == 3, "mex:r_reg", "r_reg must be [Nq x 3 x Nt] double.")
    _need(_is(pre["w_reg"], np.float64) and len(_mx_dims(pre["w_reg"])) == 2, "mex:w_reg",
          "w_reg must be [Nq x Nt] double.")
    _need(_is(pre["nearMat"], np.uint8), "mex:nearMat", "nearMat must be uint8 [Nt x Nt].")
    _need(_is(pre["self_r"], np.float64) and len(_mx_dims(pre["self_r"])) == 4, "mex:self_r",
          "self_r must be [Nq2 x 3 x NsS x Nt].")
    _need(_is(pre["self_w"], np.float64) and len(_mx_dims(pre["self_w"])) == 3, "mex:self_w",
          "self_w must be [Nq2 x NsS x Nt].")
    _need(_is(pre["self_a"], np.float64) and len(_mx_dims(pre["self_a"])) == 2, "mex:self_a",
          "self_a must be [NsS x Nt].")
    _need(_is(pre["near_r"], np.float64) and len(_mx_dims(pre["near_r"])) == 4, "mex:near_r",
          "near_r must be [Nq2 x 3 x NsN x Nt].")
    _need(_is(pre["near_w"], np.float64) and len(_mx_dims(pre["near_w"])) == 3, "mex:near_w",
          "near_w must be [Nq2 x NsN x Nt].")
    _need(_is(pre["aeqTri"], np.float64) and np.size(pre["aeqTri"]) == Nt, "mex:aeqTri", "aeqTri must be [Nt x 1].")
    d = _mx_dims(r_reg)
    _need(d[1] == 3, "mex:r_reg", "r_reg dim2 must be 3.")
    _need(d[2] == Nt, "mex:r_reg", "r_reg dim3 must be Nt.")
    d = _mx_dims(pre["self_r"])
    _need(d[1] == 3, "mex:self_r", "self_r dim2 must be 3.")
    _need(d[3] == Nt, "mex:self_r", "self_r dim4 must be Nt.")
    dn = _mx_dims(pre["near_r"])
    _need(dn[0] == d[0], "mex:near_r", "near_r Nq2 mismatch.")
    _need(dn[3] == Nt, "mex:near_r", "near_r dim4 must be Nt.")


def _port_check(pe, ge, Ne):
    _need(1 <= pe <= Ne, "mex:port", "patchEdge out of range.")
    _need(1 <= ge <= Ne, "mex:port", "groundEdge out of range.")


# ---------------------------------------------------------------------------
# Assembly-only entry points
# ---------------------------------------------------------------------------
def ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(*args, nargout=2):
    """[Z,Vrhs] = ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(V,F,E,plusTri,minusTri,plusSign,
    minusSign,rp,rm,Ap,Am,len,prepack,k,omega,mu,eps,excvec).

    Cached-quadrature FP64 assembly (ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:542-843).
    Returns Z (complex128 [Ne x Ne], Fortran order) and Vrhs (complex128 [Ne]).
    """
    _need(len(args) == 18, "mex:args", "Expected 18 inputs: V,F,E,plusTri,minusTri,plusSign,minusSign,"
                                       "rp,rm,Ap,Am,len,prepack,k,omega,mu,eps,excvec")
    _need(nargout == 2, "mex:args", "Expected 2 outputs [Z,Vrhs].")
    (V, F, E, pt, mt, ps, ms, rp, rm, Ap, Am, ln, pre, k, omega, mu, eps, exc) = args
    Nv, Nt, Ne = _check_VFE(V, F, E)
    _need(isinstance(pre, dict), "mex:prepack", "prepack must be a struct from efie_precompute_pack.")
    _need(_is(exc, np.float64) and np.size(exc) >= 4, "mex:exc",
          "excvec must be [patchEdge, groundEdge, V0, spreadRadius].")
    excv = np.asarray(exc, dtype=np.float64).reshape(-1)
    _port_check(int(excv[0]), int(excv[1]), Ne)
    for f in _PREPACK_FIELDS:
        _get_field(pre, f)
    _check_prepack_dims(pre, Nt)
    m = _Marshal()
    mesh = m.mesh(V, F, E, pt, mt, ps, ms, rp, rm, Ap, Am, ln)
    pp = m.prepack(pre, Nt)
    Z = np.zeros((Ne, Ne), dtype=np.complex128, order="F")
    Vr = np.zeros(Ne, dtype=np.complex128)
    ex = np.ascontiguousarray(excv[:4])
    nat.check(nat.lib().efie_ggassemble_zv(nat.context(), C.byref(mesh), C.byref(pp), _cscalar(k),
                                           float(_scalar(omega)), float(_scalar(mu)), _cscalar(eps),
                                           _ptr(ex, C.c_double), Z.ctypes.data, Vr.ctypes.data))
    return Z, Vr


def gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(*args, nargout=2):
    """[Z,Vrhs] = gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(V,F,E,plusTri,minusTri,plusSign,
    minusSign,rp,rm,Ap,Am,len,k,omega,mu,eps,exc), exc = [patchEdge, groundEdge,
    V0, spreadRadius, selfAlpha]: one-point centroid assembly
    (gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:125-435)."""
    _need(len(args) == 17, "mex:args", "Expected 17 inputs.")
    _need(nargout == 2, "mex:args", "Expected 2 outputs [Z,Vrhs].")
    (V, F, E, pt, mt, ps, ms, rp, rm, Ap, Am, ln, k, omega, mu, eps, exc) = args
    Nv, Nt, Ne = _check_VFE(V, F, E)
    _check_rwg_arrays(Ne, pt, mt, ps, ms, rp, rm, Ap, Am, ln)
    _need(_is(exc, np.float64) and np.size(exc) >= 5, "mex:exc",
          "exc must be double vector len>=5: [patchEdge, groundEdge, V0, spreadRadius, selfAlpha].")
    excv = np.asarray(exc, dtype=np.float64).reshape(-1)
    _port_check(int(excv[0]), int(excv[1]), Ne)
    m = _Marshal()
    mesh = m.mesh(V, F, E, pt, mt, ps, ms, rp, rm, Ap, Am, ln)
    Z = np.zeros((Ne, Ne), dtype=np.complex128, order="F")
    Vr = np.zeros(Ne, dtype=np.complex128)
    ex = np.ascontiguousarray(excv[:5])
    nat.check(nat.lib().efie_gassemble_zv(nat.context(), C.byref(mesh), _cscalar(k), float(_scalar(omega)),
                                          float(_scalar(mu)), _cscalar(eps), _ptr(ex, C.c_double),
                                          Z.ctypes.data, Vr.ctypes.data))
    return Z, Vr


def assemble_ZV_EFIE_RWG_DIFF_GPU_FAST(*args, nargout=2):
    """[Z,Vrhs] = assemble_ZV_EFIE_RWG_DIFF_GPU_FAST(rwg,prepack,k,omega,mu,eps,exc,opts).

    Struct interface of assemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:277-378:
    near_alpha comes from opts (default 0.15).  The reference reads the
    per-sub-triangle softening from a prepack field ``self_aSoft`` that
    efie_precompute_pack never writes (it writes ``self_a``); both names are
    accepted here.  rwg must carry V/F/edge as in build_rwg_interior plus the
    mesh arrays ``V`` and ``F``.
    """
    _need(len(args) == 8, "mex:args", "Expected 8 inputs: (rwg, prepack, k, omega, mu, eps, exc, opts)")
    _need(nargout == 2, "mex:args", "Expected 2 outputs: [Z, Vrhs]")
    rwg, pre, k, omega, mu, eps, exc, opts = args
    for f in ("plusTri", "minusTri", "plusSign", "minusSign"):
        _need(f in rwg, "mex:rwg", "Missing tri/sign fields")
    _need(_is(rwg["plusTri"], np.int32) and _is(rwg["minusTri"], np.int32), "mex:rwg",
          "plusTri/minusTri must be int32")
    _need(_is(rwg["plusSign"], np.int32) and _is(rwg["minusSign"], np.int32), "mex:rwg",
          "plusSign/minusSign must be int32")
    for f in ("nearMat", "r_reg", "w_reg", "aeqTri"):
        _need(f in pre, "mex:pre", "Missing prepack basic fields")
    sa_key = "self_aSoft" if "self_aSoft" in pre else "self_a"
    _need(all(f in pre for f in ("self_r", "self_w", sa_key, "near_r", "near_w")), "mex:pre",
          "Missing self/near cached fields. Use efie_prepack_for_mex(pre).")
    near_alpha = float(_scalar(opts["near_alpha"])) if isinstance(opts, dict) and "near_alpha" in opts else 0.15
    pre2 = dict(pre)
    pre2["self_a"] = pre[sa_key]
    pre2["near_alpha"] = near_alpha
    excv = np.array([exc["patchEdge"], exc["groundEdge"], exc["V0"], exc["spreadRadius"]], dtype=np.float64)
    return ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(
        rwg["V"], rwg["F"], np.asarray(rwg["edge"], dtype=np.int32), rwg["plusTri"], rwg["minusTri"],
        rwg["plusSign"], rwg["minusSign"], rwg["rp"], rwg["rm"], rwg["Ap"], rwg["Am"], rwg["len"],
        pre2, k, omega, mu, eps, excv)


# ---------------------------------------------------------------------------
# Sweeps
# ---------------------------------------------------------------------------
def sweep_opts(solver="mixed", port_model="gauss", scheme="ref", refine_tol=1e-10, refine_max_iter=30,
               timing=False, batch=0, lu_nb=0, refine="gmres", graphs=True, tile_chain=0, tile_bulk=0,
               resident_chain=0, resident_bulk=0, nfreq_hint=0, share_factors=0):
    """efie_sweep_opts: solver 'mixed'|'fp64', port_model 'gauss'|'edge',
    scheme 'ref'|'extract', refine 'gmres'|'classical' (mixed solver only),
    tile_chain / tile_bulk: tensor-core tile widths 128 | 256 (0 = tuned),
    share_factors: g >= 2 factors only the first of each group of g
    coarse-to-fine batches, the others refine with the factors of their
    nearest neighbours in it; 1: every frequency is factored; 0: automatic
    (g ~ Ne / 1200 within [2, 8])."""
    o = nat.EfieSweepOpts()
    nat.lib().efie_sweep_opts_default(C.byref(o))
    o.solver = {"fp64": nat.SOLVER_FP64, "mixed": nat.SOLVER_MIXED}[solver]
    o.port_model = {"gauss": nat.PORT_GAUSS, "edge": nat.PORT_EDGE_DIFF}[port_model]
    o.scheme = {"ref": nat.SCHEME_REF, "extract": nat.SCHEME_EXTRACT}[scheme]
    o.refine_tol = refine_tol
    o.refine_max_iter = refine_max_iter
    o.timing = 1 if timing else 0
    o.batch = int(batch)
    o.lu_nb = int(lu_nb)
    o.refine_method = {"gmres": nat.REFINE_GMRES, "classical": nat.REFINE_CLASSICAL}[refine]
    o.graphs = 1 if graphs else 0
    o.tile_chain = int(tile_chain)
    o.tile_bulk = int(tile_bulk)
    o.resident_chain = int(resident_chain)
    o.resident_bulk = int(resident_bulk)
    o.nfreq_hint = int(nfreq_hint)
    o.share_factors = int(share_factors)
    return o


def patch_sweep_fastquad_cuda(*args, nargout=2, opts=None, return_currents=False, stats=None):
    """[Zin,S11] = patch_sweep_fastquad_cuda(V,F,E,plusTri,minusTri,plusSign,minusSign,
    rp,rm,Ap,Am,len,prepack,freqs,mu,eps,patchEdge,groundEdge,V0,spreadRadius,Z0).

    Per frequency: assemble Z, solve Z I = V, Gaussian port current, Zin and
    S11 (patch_sweep_fastquad_cuda.cu:461-844).  ``opts`` (see sweep_opts)
    selects the solver; the default is the mixed-precision solver with FP64
    refinement to a relative residual of 1e-10.  With ``return_currents`` the
    solution currents I [Ne x Nf] are returned as a third output.
    """
    _need(len(args) == 21, "mex:args", "Expected 21 inputs.")
    _need(nargout == 2, "mex:args", "Expected 2 outputs [Zin,S11].")
    (V, F, E, pt, mt, ps, ms, rp, rm, Ap, Am, ln, pre, freqs, mu, eps, pe, ge, V0, spread, Z0) = args
    Nv, Nt, Ne = _check_VFE(V, F, E)
    _need(_is(freqs, np.float64), "mex:freqs", "freqs must be double vector.")
    _need(isinstance(pre, dict), "mex:prepack", "prepack must be struct.")
    pe = int(_scalar(pe))
    ge = int(_scalar(ge))
    _port_check(pe, ge, Ne)
    for f in _PREPACK_FIELDS:
        _get_field(pre, f)
    m = _Marshal()
    mesh = m.mesh(V, F, E, pt, mt, ps, ms, rp, rm, Ap, Am, ln)
    pp = m.prepack(pre, Nt)
    fr = _f64(freqs)
    Nf = fr.size
    Zin = np.zeros(Nf, dtype=np.complex128)
    S11 = np.zeros(Nf, dtype=np.complex128)
    I = np.zeros((Ne, Nf), dtype=np.complex128, order="F") if return_currents else None
    st = nat.EfieSweepStats()
    o = opts if opts is not None else sweep_opts()
    nat.check(nat.lib().efie_patch_sweep_fastquad(
        nat.context(), C.byref(mesh), C.byref(pp), _ptr(fr, C.c_double), Nf, float(_scalar(mu)), _cscalar(eps),
        pe, ge, float(_scalar(V0)), float(_scalar(spread)), float(_scalar(Z0)), C.byref(o),
        Zin.ctypes.data, S11.ctypes.data, I.ctypes.data if I is not None else None, C.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return (Zin, S11, I) if return_currents else (Zin, S11)


def patch_sweep_cuda(*args, nargout=2, opts=None, stats=None):
    """[Zin,S11] = patch_sweep_cuda(V,F,edge,plusTri,minusTri,plusSign,minusSign,rp,rm,
    Ap,Am,len,freqs,mu,eps,patchEdge,groundEdge,V0,spreadRadius,Z0).

    Centroid assembly with selfAlpha = 0.20 and the edge-difference port
    current Iport = I(patchEdge) - I(groundEdge) (patch_sweep_cuda.cu:172-527).
    """
    _need(len(args) == 20, "mex:args", "Expected 20 inputs.")
    _need(nargout == 2, "mex:args", "Expected 2 outputs [Zin,S11].")
    (V, F, E, pt, mt, ps, ms, rp, rm, Ap, Am, ln, freqs, mu, eps, pe, ge, V0, spread, Z0) = args
    Nv, Nt, Ne = _check_VFE(V, F, E, "mex:edge", "edge must be [Ne x 2] int32.")
    _check_rwg_arrays(Ne, pt, mt, ps, ms, rp, rm, Ap, Am, ln)
    _need(_is(freqs, np.float64), "mex:freqs", "freqs must be double vector.")
    pe = int(_scalar(pe))
    ge = int(_scalar(ge))
    _port_check(pe, ge, Ne)
    m = _Marshal()
    mesh = m.mesh(V, F, E, pt, mt, ps, ms, rp, rm, Ap, Am, ln)
    fr = _f64(freqs)
    Nf = fr.size
    Zin = np.zeros(Nf, dtype=np.complex128)
    S11 = np.zeros(Nf, dtype=np.complex128)
    st = nat.EfieSweepStats()
    o = opts if opts is not None else sweep_opts()
    nat.check(nat.lib().efie_patch_sweep_centroid(
        nat.context(), C.byref(mesh), _ptr(fr, C.c_double), Nf, float(_scalar(mu)), _cscalar(eps), pe, ge,
        float(_scalar(V0)), float(_scalar(spread)), float(_scalar(Z0)), C.byref(o), Zin.ctypes.data,
        S11.ctypes.data, None, C.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return Zin, S11


def _precompute_opts(opts):
    """efie_precompute_opts with efie_precompute.m's defaults (:5, :45-48)."""
    return nat.EfiePrecomputeOpts(int(opts["quad_order"]), int(opts.get("near_order", 4)),
                                  int(opts.get("self_subdiv", 2)), int(opts.get("near_subdiv", 2)),
                                  float(opts["near_sing_eps"]), float(opts.get("self_alpha", 0.20)),
                                  float(opts.get("near_alpha", 0.15)))


class SweepPlan:
    """Geometry uploaded once; ``run(freqs)`` sweeps with device-resident data.

    Arguments are those of patch_sweep_fastquad_cuda minus ``freqs``.  With
    ``pre=None`` and ``precompute`` (the options of efie_precompute, e.g.
    ``quad_order``, ``near_sing_eps``, ...) the prepack of the reference
    scheme is computed on the GPU from V/F (no host nearMat).
    """

    def __init__(self, V, F, E, pt, mt, ps, ms, rp, rm, Ap, Am, ln, pre, mu, eps, pe, ge, V0, spread, Z0,
                 opts=None, rule_order=0, precompute=None, ctx=None):
        Nv, Nt, Ne = _check_VFE(V, F, E)
        self.Ne = Ne
        self._m = _Marshal()
        self._mesh = self._m.mesh(V, F, E, pt, mt, ps, ms, rp, rm, Ap, Am, ln)
        self._pp = self._m.prepack(pre, Nt) if pre is not None else None
        if opts is None:
            from .autotune import tuned_opts
            t = tuned_opts(Ne)
            opts = (sweep_opts(batch=t[0], lu_nb=t[1], tile_chain=t[2], tile_bulk=t[3], resident_chain=t[4],
                               resident_bulk=t[5], share_factors=t[6]) if t else sweep_opts())
        self.opts = opts
        h = C.c_void_p()
        cx = ctx if ctx is not None else nat.context()
        if pre is None and precompute is not None:
            po = _precompute_opts(precompute)
            nat.check(nat.lib().efie_plan_create_mesh(
                cx, C.byref(self._mesh), C.byref(po), float(_scalar(mu)), _cscalar(eps),
                int(_scalar(pe)), int(_scalar(ge)), float(_scalar(V0)), float(_scalar(spread)), float(_scalar(Z0)),
                C.byref(self.opts), C.byref(h)))
        else:
            nat.check(nat.lib().efie_plan_create(
                cx, C.byref(self._mesh), C.byref(self._pp) if self._pp is not None else None,
                float(_scalar(mu)), _cscalar(eps), int(_scalar(pe)), int(_scalar(ge)), float(_scalar(V0)),
                float(_scalar(spread)), float(_scalar(Z0)), C.byref(self.opts), int(rule_order), C.byref(h)))
        self._h = h
        if ctx is None:
            nat.register_plan(self)   # plans on their own contexts are closed by their owner

    def run(self, freqs, return_currents=False):
        fr = _f64(freqs)
        Nf = fr.size
        Zin = np.zeros(Nf, dtype=np.complex128)
        S11 = np.zeros(Nf, dtype=np.complex128)
        I = np.zeros((self.Ne, Nf), dtype=np.complex128, order="F") if return_currents else None
        st = nat.EfieSweepStats()
        nat.check(nat.lib().efie_plan_run(self._h, _ptr(fr, C.c_double), Nf, Zin.ctypes.data, S11.ctypes.data,
                                          I.ctypes.data if I is not None else None, C.byref(st)))
        self.stats = st.as_dict()
        return (Zin, S11, I) if return_currents else (Zin, S11)

    def set_timing(self, on):
        """Per-kernel-class event timing of later runs (eager launches) or not
        (the factorization replays a CUDA graph)."""
        nat.check(nat.lib().efie_plan_set_timing(self._h, 1 if on else 0))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            nat.lib().efie_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Boundary-data producers (MATLAB-side in the reference)
# ---------------------------------------------------------------------------
def make_patch_with_ground_mesh(Lp, Wp, Lg, Wg, h, Np_x, Np_y, Ng_x, Ng_y, vertex_order="reference"):
    """[V,F,patchFaceIdx,groundFaceIdx] = make_patch_with_ground_mesh(...) (make_patch_with_ground_mesh.m:1-46).

    ``vertex_order='reference'`` reproduces the reference numbering exactly
    (y-fastest vertices, x-fastest faces); ``'grid'`` numbers the vertices
    x-fastest so that each face is half of a grid rectangle.
    """
    Nv = (Np_x + 1) * (Np_y + 1) + (Ng_x + 1) * (Ng_y + 1)
    Nt = 2 * (Np_x * Np_y + Ng_x * Ng_y)
    V = np.zeros((Nv, 3), dtype=np.float64, order="F")
    F = np.zeros((Nt, 3), dtype=np.int32, order="F")
    vo = {"reference": 0, "grid": 1}[vertex_order]
    nat.check(nat.lib().efie_make_patch_with_ground_mesh(
        float(Lp), float(Wp), float(Lg), float(Wg), float(h), int(Np_x), int(Np_y), int(Ng_x), int(Ng_y), vo,
        V.ctypes.data_as(nat.c_double_p), F.ctypes.data_as(nat.c_int32_p)))
    npf = 2 * Np_x * Np_y
    return V, F, np.arange(1, npf + 1), npf + np.arange(1, Nt - npf + 1)


def build_rwg_interior(mesh):
    """rwg = build_rwg_interior(mesh) (build_rwg_interior.m:1-103), mesh = {'V':..., 'F':...}.

    Index fields are int32 (the casts main_patch_gpu_mex_sweep_l.m:28-32 apply).
    """
    V = np.asfortranarray(np.asarray(mesh["V"], dtype=np.float64))
    F = np.asfortranarray(np.asarray(mesh["F"], dtype=np.int32))
    Nv, Nt = V.shape[0], F.shape[0]
    L = nat.lib()
    Ne = C.c_int32()
    vp = V.ctypes.data_as(nat.c_double_p)
    fp = F.ctypes.data_as(nat.c_int32_p)
    nat.check(L.efie_build_rwg_interior(Nv, vp, Nt, fp, 0, C.byref(Ne), *([None] * 12)))
    n = Ne.value
    out = dict(edge=np.zeros((n, 2), np.int32, order="F"), plusTri=np.zeros(n, np.int32),
               minusTri=np.zeros(n, np.int32), plusSign=np.zeros(n, np.int32), minusSign=np.zeros(n, np.int32),
               rp=np.zeros((n, 3), order="F"), rm=np.zeros((n, 3), order="F"), Ap=np.zeros(n), Am=np.zeros(n),
               len=np.zeros(n), center=np.zeros((n, 3), order="F"), zSign=np.zeros(n, np.int32))
    i32 = lambda a: a.ctypes.data_as(nat.c_int32_p)
    f64 = lambda a: a.ctypes.data_as(nat.c_double_p)
    nat.check(L.efie_build_rwg_interior(
        Nv, vp, Nt, fp, n, C.byref(Ne), i32(out["edge"]), i32(out["plusTri"]), i32(out["minusTri"]),
        i32(out["plusSign"]), i32(out["minusSign"]), f64(out["rp"]), f64(out["rm"]), f64(out["Ap"]),
        f64(out["Am"]), f64(out["len"]), f64(out["center"]), i32(out["zSign"])))
    out["Ne"] = n
    return out


def build_patch_design_gpu(Lp, Wp, Lg, Wg, h, Np_x, Np_y, Ng_x, Ng_y, feed=(0.0, -7e-3), vertex_order="reference",
                           ctx=None):
    """Mesh, RWG topology and port edges of a two-plate design built on the GPU
    (make_patch_with_ground_mesh.m, build_rwg_interior.m,
    pick_port_edge_by_point_and_layer.m at (feed, +-h/2)).  Returns
    (V, F, rwg, patchEdge, groundEdge) exactly as the host producers do."""
    vo = {"reference": 0, "grid": 1}[vertex_order]
    L = nat.lib()
    h_ = C.c_void_p()
    fd = np.ascontiguousarray(np.asarray(feed, dtype=np.float64).reshape(2))
    nat.check(L.efie_design_build(ctx if ctx is not None else nat.context(), float(Lp), float(Wp), float(Lg), float(Wg), float(h), int(Np_x),
                                  int(Np_y), int(Ng_x), int(Ng_y), vo, fd.ctypes.data_as(nat.c_double_p),
                                  C.byref(h_)))
    try:
        n = [C.c_int32() for _ in range(5)]
        nat.check(L.efie_design_sizes(h_, *[C.byref(x) for x in n]))
        Nv, Nt, Ne, pe, ge = (x.value for x in n)
        V = np.zeros((Nv, 3), np.float64, order="F")
        F = np.zeros((Nt, 3), np.int32, order="F")
        r = dict(edge=np.zeros((Ne, 2), np.int32, order="F"), plusTri=np.zeros(Ne, np.int32),
                 minusTri=np.zeros(Ne, np.int32), plusSign=np.zeros(Ne, np.int32), minusSign=np.zeros(Ne, np.int32),
                 rp=np.zeros((Ne, 3), order="F"), rm=np.zeros((Ne, 3), order="F"), Ap=np.zeros(Ne),
                 Am=np.zeros(Ne), len=np.zeros(Ne), center=np.zeros((Ne, 3), order="F"),
                 zSign=np.zeros(Ne, np.int32))
        i32 = lambda a: a.ctypes.data_as(nat.c_int32_p)
        f64 = lambda a: a.ctypes.data_as(nat.c_double_p)
        nat.check(L.efie_design_read(h_, f64(V), i32(F), i32(r["edge"]), i32(r["plusTri"]), i32(r["minusTri"]),
                                     i32(r["plusSign"]), i32(r["minusSign"]), f64(r["rp"]), f64(r["rm"]),
                                     f64(r["Ap"]), f64(r["Am"]), f64(r["len"]), f64(r["center"]),
                                     i32(r["zSign"])))
        r["Ne"] = Ne
    finally:
        L.efie_design_destroy(h_)
    return V, F, r, pe, ge


def pick_port_edge_by_point_and_layer(rwg, p, layerSign):
    """eidx = pick_port_edge_by_point_and_layer(rwg,p,layerSign) (1-based; first minimum)."""
    c = np.asfortranarray(np.asarray(rwg["center"], dtype=np.float64))
    z = np.ascontiguousarray(np.asarray(rwg["zSign"], dtype=np.int32))
    pp = np.ascontiguousarray(np.asarray(p, dtype=np.float64).reshape(3))
    e = C.c_int32()
    nat.check(nat.lib().efie_pick_port_edge(c.shape[0], c.ctypes.data_as(nat.c_double_p),
                                            z.ctypes.data_as(nat.c_int32_p), pp.ctypes.data_as(nat.c_double_p),
                                            int(layerSign), C.byref(e)))
    return e.value


def quad_rule_size(order):
    return int(nat.lib().efie_quad_rule_size(int(order)))


def efie_precompute_pack_gpu(mesh, opts):
    """efie_precompute_pack computed on the GPU (same outputs, bit for bit)."""
    return efie_precompute_pack(mesh, opts, gpu=True)


def efie_precompute_pack(mesh, opts, gpu=False):
    """prepack = efie_precompute_pack(efie_precompute(mesh,opts),opts) in one call
    (efie_precompute.m:1-97, efie_precompute_pack.m:1-59), with the same option
    defaults (near_order 4, self_subdiv 2, self_alpha 0.20, near_subdiv 2,
    near_alpha 0.15)."""
    V = np.asfortranarray(np.asarray(mesh["V"], dtype=np.float64))
    F = np.asfortranarray(np.asarray(mesh["F"], dtype=np.int32))
    Nv, Nt = V.shape[0], F.shape[0]
    o = _precompute_opts(opts)
    Nq, Nq2 = quad_rule_size(o.quad_order), quad_rule_size(o.near_order)
    NsS, NsN = 4 ** o.self_subdiv, 4 ** o.near_subdiv
    pre = dict(r_reg=np.zeros((Nq, 3, Nt), order="F"), w_reg=np.zeros((Nq, Nt), order="F"),
               nearMat=np.zeros((Nt, Nt), np.uint8, order="F"),
               self_r=np.zeros((Nq2, 3, NsS, Nt), order="F"), self_w=np.zeros((Nq2, NsS, Nt), order="F"),
               self_a=np.zeros((NsS, Nt), order="F"), near_r=np.zeros((Nq2, 3, NsN, Nt), order="F"),
               near_w=np.zeros((Nq2, NsN, Nt), order="F"), aeqTri=np.zeros(Nt))
    f64 = lambda a: a.ctypes.data_as(nat.c_double_p)
    pp = nat.EfiePrepack(Nt, Nq, Nq2, NsS, NsN, f64(pre["r_reg"]), f64(pre["w_reg"]),
                         pre["nearMat"].ctypes.data_as(nat.c_uint8_p), f64(pre["self_r"]), f64(pre["self_w"]),
                         f64(pre["self_a"]), f64(pre["near_r"]), f64(pre["near_w"]), f64(pre["aeqTri"]), 0.0, 0.0)
    if gpu:
        nat.check(nat.lib().efie_precompute_pack_gpu(nat.context(), Nv, V.ctypes.data_as(nat.c_double_p), Nt,
                                                     F.ctypes.data_as(nat.c_int32_p), C.byref(o), C.byref(pp)))
    else:
        nat.check(nat.lib().efie_precompute_pack(Nv, V.ctypes.data_as(nat.c_double_p), Nt,
                                                 F.ctypes.data_as(nat.c_int32_p), C.byref(o), C.byref(pp)))
    pre["near_alpha"] = pp.near_alpha
    pre["self_alpha"] = pp.self_alpha
    return pre
