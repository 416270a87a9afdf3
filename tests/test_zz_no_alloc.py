"""GPU test of efie_gassemble_zv_noalloc, the centroid assembly that allocates
no device memory (for callers that cannot call cudaMalloc: processes held to
a device-memory budget fixed at start-up, hosts that own every device
buffer).  It is called through the C ABI on device buffers that the
test owns, twice in a row (the second call must not see the first call's
scratch contents), and compared with the allocating entry point
efie_gassemble_zv on the same inputs: |dZ| <= 1e-13 max|Z|, |dV| <= 1e-14 max|V|.
This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process."""
import ctypes as C
import importlib

import numpy as np
import pytest

import efie_oracle as eo
from conftest import small_design, config1_design

pytestmark = pytest.mark.gpu


def _noalloc(p, k, omega, self_alpha, edit=None, spread=None):
    torch = pytest.importorskip("torch")
    nat = importlib.import_module("matlab-cuda-efief-vs-cpu_b200._native")
    r = p["rwg"]
    d = p["design"]
    dev = torch.device("cuda", 0)

    def tdev(a, dt):
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=dt).reshape(-1, order="F"))).to(dev)

    arrs = dict(V=p["V"], F=p["F"], E=r["edge"], plusTri=r["plusTri"])
    if edit:
        arrs = {key: np.array(a, copy=True) for key, a in arrs.items()}
        edit(arrs)
    bufs = [tdev(arrs["V"], np.float64), tdev(arrs["F"], np.int32), tdev(arrs["E"], np.int32),
            tdev(arrs["plusTri"], np.int32), tdev(r["minusTri"], np.int32), tdev(r["plusSign"], np.int32),
            tdev(r["minusSign"], np.int32), tdev(r["rp"], np.float64), tdev(r["rm"], np.float64),
            tdev(r["Ap"], np.float64), tdev(r["Am"], np.float64), tdev(r["len"], np.float64)]
    Ne = r["Ne"]
    Z = torch.full((2 * Ne * Ne,), float("nan"), dtype=torch.float64, device=dev)
    V = torch.full((2 * Ne,), float("nan"), dtype=torch.float64, device=dev)
    exc = np.array([p["patchEdge"], p["groundEdge"], d.V0, p["spread"] if spread is None else spread, self_alpha],
                   dtype=np.float64)
    stream = torch.cuda.current_stream(dev)
    kk = complex(k)
    ee = complex(d.eps)
    st = nat.lib().efie_gassemble_zv_noalloc(
        0, stream.cuda_stream, p["V"].shape[0], p["F"].shape[0], Ne, *[b.data_ptr() for b in bufs],
        nat.c128(kk.real, kk.imag), omega, d.mu, nat.c128(ee.real, ee.imag),
        exc.ctypes.data_as(C.POINTER(C.c_double)), Z.data_ptr(), V.data_ptr())
    if edit is not None or spread is not None:
        return nat.lib().efie_status_id(st).decode()
    nat.check(st)
    Zc = Z.cpu().numpy().view(np.complex128).reshape(Ne, Ne, order="F")
    Vc = V.cpu().numpy().view(np.complex128)
    return Zc, Vc


def _alloc(p, k, omega, self_alpha):
    m = importlib.import_module("matlab-cuda-efief-vs-cpu_b200")
    r = p["rwg"]
    d = p["design"]
    exc = np.array([p["patchEdge"], p["groundEdge"], d.V0, p["spread"], self_alpha], dtype=np.float64)
    return m.gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(
        p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
        r["Ap"], r["Am"], r["len"], k, omega, d.mu, d.eps, exc)


def test_noalloc_matches_allocating_entry_point_twice():
    # a larger problem first, then a smaller one: the second call runs on
    # scratch that still holds the first call's data
    for design, f, sa in ((config1_design("grid"), 2.4e9, 0.2), (small_design("reference"), 2.9e9, 0.25)):
        p = eo.build_problem(design)
        omega, k, _, _ = eo.physics(f, design.mu, design.eps)
        Zn, Vn = _noalloc(p, k, omega, sa)
        Za, Va = _alloc(p, k, omega, sa)
        assert np.all(np.isfinite(Zn)) and np.all(np.isfinite(Vn))
        assert np.abs(Zn - Za).max() <= 1e-13 * np.abs(Za).max()
        assert np.abs(Vn - Va).max() <= 1e-14 * np.abs(Va).max()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    nat = importlib.import_module("matlab-cuda-efief-vs-cpu_b200._native")
    exc = np.array([1, 1, 1.0, 1e-3, 0.2])
    st = nat.lib().efie_gassemble_zv_noalloc(
        0, None, 3, 1, nat.NOALLOC_MAX_NE + 1, *([None] * 12), nat.c128(1.0, 0.0), 1.0, 1.0, nat.c128(1.0, 0.0),
        exc.ctypes.data_as(C.POINTER(C.c_double)), None, None)
    assert nat.lib().efie_status_id(st) == b"mex:args"
    assert b"16384" in nat.lib().efie_last_error()


def test_noalloc_reports_device_side_index_errors_then_recovers():
    """Inputs whose errors only the kernels can see -- a face or an edge that
    names a vertex past Nv, a plusTri past Nt, a zero spreadRadius (no
    Gaussian port weights) -- come back as the reference's error identifiers.
    The kernels check every index before they use it, so nothing outside the
    buffers is read.  The status word is cleared by every call: a valid call
    right after the failures matches the allocating entry point."""
    design = small_design("grid")
    p = eo.build_problem(design)
    omega, k, _, _ = eo.physics(2.5e9, design.mu, design.eps)
    Nv, Nt = p["V"].shape[0], p["F"].shape[0]

    def bad_face(a):
        a["F"][3, 1] = Nv + 1

    def bad_edge(a):
        a["E"][5, 0] = Nv + 7

    def bad_tri(a):
        a["plusTri"][2] = Nt + 1

    assert _noalloc(p, k, omega, 0.2, edit=bad_face) == "mex:F"
    assert _noalloc(p, k, omega, 0.2, edit=bad_edge) == "mex:E"
    assert _noalloc(p, k, omega, 0.2, edit=bad_tri) == "mex:rwg"
    assert _noalloc(p, k, omega, 0.2, spread=0.0) == "mex:rhs"
    Zn, Vn = _noalloc(p, k, omega, 0.2)
    Za, Va = _alloc(p, k, omega, 0.2)
    assert np.abs(Zn - Za).max() <= 1e-13 * np.abs(Za).max()
    assert np.abs(Vn - Va).max() <= 1e-14 * np.abs(Va).max()
