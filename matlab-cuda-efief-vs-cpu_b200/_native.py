"""ctypes binding of libefie_b200.so (the C ABI declared in include/efie_b200.h).

The library is built in-tree by ``build.py``; there is no fallback: if the
shared object is missing or no CUDA device is present, calls raise.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os
import weakref

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libefie_b200.so")

c_double_p = C.POINTER(C.c_double)
c_int32_p = C.POINTER(C.c_int32)
c_uint8_p = C.POINTER(C.c_uint8)


class c128(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class EfieMesh(C.Structure):
    _fields_ = [("Nv", C.c_int32), ("Nt", C.c_int32), ("Ne", C.c_int32),
                ("V", c_double_p), ("F", c_int32_p), ("E", c_int32_p),
                ("plusTri", c_int32_p), ("minusTri", c_int32_p),
                ("plusSign", c_int32_p), ("minusSign", c_int32_p),
                ("rp", c_double_p), ("rm", c_double_p),
                ("Ap", c_double_p), ("Am", c_double_p), ("len", c_double_p)]


class EfiePrepack(C.Structure):
    _fields_ = [("Nt", C.c_int32), ("Nq", C.c_int32), ("Nq2", C.c_int32),
                ("NsS", C.c_int32), ("NsN", C.c_int32),
                ("r_reg", c_double_p), ("w_reg", c_double_p), ("nearMat", c_uint8_p),
                ("self_r", c_double_p), ("self_w", c_double_p), ("self_a", c_double_p),
                ("near_r", c_double_p), ("near_w", c_double_p), ("aeqTri", c_double_p),
                ("near_alpha", C.c_double), ("self_alpha", C.c_double)]


class EfieSweepOpts(C.Structure):
    _fields_ = [("solver", C.c_int32), ("port_model", C.c_int32), ("scheme", C.c_int32),
                ("refine_tol", C.c_double), ("refine_max_iter", C.c_int32),
                ("lu_nb", C.c_int32), ("timing", C.c_int32), ("batch", C.c_int32),
                ("refine_method", C.c_int32), ("graphs", C.c_int32), ("tile_chain", C.c_int32),
                ("tile_bulk", C.c_int32), ("resident_chain", C.c_int32), ("resident_bulk", C.c_int32),
                ("nfreq_hint", C.c_int32), ("share_factors", C.c_int32)]


KERNEL_CLASSES = ("quad", "nearself", "gather", "gemm", "panel", "trsv", "residual", "other")


class EfieSweepStats(C.Structure):
    _fields_ = [("n_freq", C.c_int32), ("refine_iters_max", C.c_int32),
                ("n_fp64_fallback", C.c_int32), ("max_relres", C.c_double),
                ("ms_assemble", C.c_double), ("ms_factor", C.c_double), ("ms_solve", C.c_double),
                ("n_launches", C.c_int32),
                ("class_launches", C.c_int32 * 8), ("class_ms", C.c_double * 8), ("class_work", C.c_double * 8),
                ("n_wait_timeouts", C.c_int32), ("n_zero_pivots", C.c_int32),
                ("n_shared_factors", C.c_int32)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if not f.startswith("class_")}
        d["classes"] = {name: dict(launches=self.class_launches[i], ms=self.class_ms[i], work=self.class_work[i])
                        for i, name in enumerate(KERNEL_CLASSES)}
        return d


class EfiePrecomputeOpts(C.Structure):
    _fields_ = [("quad_order", C.c_int32), ("near_order", C.c_int32),
                ("self_subdiv", C.c_int32), ("near_subdiv", C.c_int32),
                ("near_sing_eps", C.c_double), ("self_alpha", C.c_double),
                ("near_alpha", C.c_double)]


SOLVER_FP64, SOLVER_MIXED = 0, 1
PORT_GAUSS, PORT_EDGE_DIFF = 0, 1
SCHEME_REF, SCHEME_EXTRACT = 0, 1
REFINE_GMRES, REFINE_CLASSICAL = 0, 1
QUAD_DUNAVANT7 = -7

# Every exported symbol of include/efie_b200.h with (restype, argtypes).
_P = C.c_void_p
SIGNATURES = {
    "efie_status_id": (C.c_char_p, [C.c_int]),
    "efie_last_error": (C.c_char_p, []),
    "efie_ctx_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "efie_ctx_destroy": (None, [_P]),
    "efie_ctx_set_stream": (C.c_int, [_P, _P]),
    "efie_ggassemble_zv": (C.c_int, [_P, C.POINTER(EfieMesh), C.POINTER(EfiePrepack), c128, C.c_double,
                                     C.c_double, c128, c_double_p, _P, _P]),
    "efie_gassemble_zv": (C.c_int, [_P, C.POINTER(EfieMesh), c128, C.c_double, C.c_double, c128,
                                    c_double_p, _P, _P]),
    "efie_sweep_opts_default": (None, [C.POINTER(EfieSweepOpts)]),
    "efie_patch_sweep_fastquad": (C.c_int, [_P, C.POINTER(EfieMesh), C.POINTER(EfiePrepack), c_double_p,
                                            C.c_int32, C.c_double, c128, C.c_int32, C.c_int32, C.c_double,
                                            C.c_double, C.c_double, C.POINTER(EfieSweepOpts), _P, _P, _P,
                                            C.POINTER(EfieSweepStats)]),
    "efie_patch_sweep_centroid": (C.c_int, [_P, C.POINTER(EfieMesh), c_double_p, C.c_int32, C.c_double,
                                            c128, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                            C.POINTER(EfieSweepOpts), _P, _P, _P, C.POINTER(EfieSweepStats)]),
    "efie_plan_create": (C.c_int, [_P, C.POINTER(EfieMesh), C.POINTER(EfiePrepack), C.c_double, c128,
                                   C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                   C.POINTER(EfieSweepOpts), C.c_int32, C.POINTER(_P)]),
    "efie_plan_run": (C.c_int, [_P, c_double_p, C.c_int32, _P, _P, _P, C.POINTER(EfieSweepStats)]),
    "efie_plan_destroy": (None, [_P]),
    "efie_plan_set_timing": (C.c_int, [_P, C.c_int32]),
    "efie_make_patch_with_ground_mesh": (C.c_int, [C.c_double] * 5 + [C.c_int32] * 5 + [c_double_p, c_int32_p]),
    "efie_build_rwg_interior": (C.c_int, [C.c_int32, c_double_p, C.c_int32, c_int32_p, C.c_int32, c_int32_p,
                                          c_int32_p, c_int32_p, c_int32_p, c_int32_p, c_int32_p,
                                          c_double_p, c_double_p, c_double_p, c_double_p, c_double_p,
                                          c_double_p, c_int32_p]),
    "efie_pick_port_edge": (C.c_int, [C.c_int32, c_double_p, c_int32_p, c_double_p, C.c_int32, c_int32_p]),
    "efie_quad_rule_size": (C.c_int32, [C.c_int32]),
    "efie_precompute_pack": (C.c_int, [C.c_int32, c_double_p, C.c_int32, c_int32_p,
                                       C.POINTER(EfiePrecomputeOpts), C.POINTER(EfiePrepack)]),
    "efie_design_build": (C.c_int, [_P] + [C.c_double] * 5 + [C.c_int32] * 5 + [c_double_p, C.POINTER(_P)]),
    "efie_design_sizes": (C.c_int, [_P] + [c_int32_p] * 5),
    "efie_design_read": (C.c_int, [_P, c_double_p, c_int32_p, c_int32_p, c_int32_p, c_int32_p, c_int32_p, c_int32_p,
                                   c_double_p, c_double_p, c_double_p, c_double_p, c_double_p, c_double_p,
                                   c_int32_p]),
    "efie_design_destroy": (None, [_P]),
    "efie_precompute_pack_gpu": (C.c_int, [_P, C.c_int32, c_double_p, C.c_int32, c_int32_p,
                                           C.POINTER(EfiePrecomputeOpts), C.POINTER(EfiePrepack)]),
    "efie_plan_create_mesh": (C.c_int, [_P, C.POINTER(EfieMesh), C.POINTER(EfiePrecomputeOpts), C.c_double, c128,
                                        C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                        C.POINTER(EfieSweepOpts), C.POINTER(_P)]),
    "efie_lu_selftest": (C.c_int, [_P, C.c_int32, _P, C.c_int32, _P]),
    "efie_debug_disable_tensor_cores": (None, [C.c_int]),
    "efie_debug_disable_symmetric_lu": (None, [C.c_int]),
    "efie_debug_set_selftest_panel": (None, [C.c_int]),
    "efie_debug_set_selftest_tiles": (None, [C.c_int, C.c_int, C.c_int]),
    "efie_debug_disable_warm_start": (None, [C.c_int]),
    "efie_debug_set_wait_test": (C.c_int, [C.c_int32, C.c_int64]),
    "efie_gassemble_zv_noalloc": (C.c_int, [C.c_int, _P, C.c_int32, C.c_int32, C.c_int32] + [_P] * 12 +
                                  [c128, C.c_double, C.c_double, c128, c_double_p, _P, _P]),
    "efie_mlp_config_default": (None, [_P]),
    "efie_adam_opts_default": (None, [_P]),
    "efie_mlp_create": (C.c_int, [_P, _P, C.POINTER(_P)]),
    "efie_mlp_destroy": (None, [_P]),
    "efie_mlp_num_params": (C.c_int64, [_P]),
    "efie_mlp_get_params": (C.c_int, [_P, _P]),
    "efie_mlp_set_params": (C.c_int, [_P, _P]),
    "efie_mlp_forward": (C.c_int, [_P, _P, C.c_int32, _P]),
    "efie_mlp_loss_grad": (C.c_int, [_P, _P, _P, C.c_int32, _P, _P]),
    "efie_mlp_train": (C.c_int, [_P, _P, _P, C.c_int32, _P, _P]),
}


class EfieMlpConfig(C.Structure):
    _fields_ = [("n_in", C.c_int32), ("n_hidden", C.c_int32), ("n_layers", C.c_int32), ("n_out", C.c_int32),
                ("seed", C.c_uint64)]


class EfieAdamOpts(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("weight_decay", C.c_float), ("batch", C.c_int32), ("epochs", C.c_int32), ("seed", C.c_uint64)]

NOALLOC_MAX_NE = 16384
NOALLOC_MAX_NT = 16384

_lib = None


def lib():
    """Load libefie_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libefie_b200.so is not built: run __graft_entry__.build() "
                               "or python matlab-cuda-efief-vs-cpu_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class MexError(RuntimeError):
    """Error carrying the reference's mexErrMsgIdAndTxt identifier."""

    def __init__(self, identifier, message):
        super().__init__("%s: %s" % (identifier, message))
        self.identifier = identifier
        self.message = message


def check(status):
    if status != 0:
        L = lib()
        raise MexError(L.efie_status_id(status).decode(), L.efie_last_error().decode())


_ctx = None
_plans = weakref.WeakSet()   # live plans: destroyed before their context


def context(device=0):
    """Process-wide context (created on first use, destroyed at exit like mexAtExit)."""
    global _ctx
    if _ctx is None:
        h = C.c_void_p()
        check(lib().efie_ctx_create(device, C.byref(h)))
        _ctx = h
        atexit.register(_destroy_ctx)
    return _ctx


def new_context(device=0):
    """A further context on `device` (its own CUDA stream and solver handle),
    for a host thread of its own; release it with destroy_context after the
    plans created on it."""
    h = C.c_void_p()
    check(lib().efie_ctx_create(device, C.byref(h)))
    return h


def destroy_context(h):
    if h is not None and h.value:
        lib().efie_ctx_destroy(h)


def register_plan(plan):
    _plans.add(plan)


def _destroy_ctx():
    global _ctx
    for p in list(_plans):
        p.close()
    if _ctx is not None and _lib is not None:
        _lib.efie_ctx_destroy(_ctx)
    _ctx = None
