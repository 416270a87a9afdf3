"""GPU parity of the assembly entry points (through the C ABI) against the
FP64 oracle and against the reference's own CUDA code (oracle/_ref).
Tolerance: max |Z - Z_ref| <= 1e-12 * max |Z_ref| (FP64 vs FP64, different
summation order)."""
import numpy as np
import pytest

import efie_oracle as eo
import oracle_c as oc
from conftest import pkg, small_design, config1_design

pytestmark = pytest.mark.gpu
TOL_Z = 1e-12


def _gg(p, k, omega):
    m = pkg()
    r = p["rwg"]
    d = p["design"]
    exc = np.array([p["patchEdge"], p["groundEdge"], d.V0, p["spread"]], dtype=np.float64)
    return m.ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(
        p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
        r["Ap"], r["Am"], r["len"], p["prepack"], k, omega, d.mu, d.eps, exc)


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


DESIGNS = {
    "small_grid": lambda: small_design("grid"),
    "small_reference_order": lambda: small_design("reference"),
    "small_accurate": lambda: small_design("grid", opts=eo.DEFAULT_OPTS_ACCURATE, npx=3, npy=2, ngx=4, ngy=4),
    "reference_sweep_538": eo.reference_sweep_design,
    "config1_1074": lambda: config1_design("grid"),
}


@pytest.mark.parametrize("name", list(DESIGNS))
def test_ggassemble_matches_oracle(name):
    d = DESIGNS[name]()
    p = eo.build_problem(d)
    omega, k, _, _ = eo.physics(d.freqs[len(d.freqs) // 2], d.mu, d.eps)
    Z, V = _gg(p, k, omega)
    Zo = oc.assemble_z(p["rwg"], p["prepack"], k, omega, d.mu, d.eps)
    assert _rel(Z, Zo) < TOL_Z
    assert np.abs(V.real - p["b"]).max() <= 1e-14 * np.abs(p["b"]).max() and np.all(V.imag == 0)


def test_ggassemble_matches_reference_cuda():
    ref_mex = pytest.importorskip("ref_mex")
    d = eo.reference_sweep_design()
    p = eo.build_problem(d)
    omega, k, _, _ = eo.physics(1.2e9, d.mu, d.eps)
    Zr, Vr = ref_mex.ggassemble(p, k, omega, d.mu, d.eps)
    Z, V = _gg(p, k, omega)
    assert _rel(Z, Zr) < TOL_Z
    assert np.array_equal(V, Vr)


def test_lossy_complex_k_and_half_rwg():
    """Complex k (lossy eps) and an edge with one triangle missing (t = 0)."""
    d = small_design("grid")
    d.eps = eo.EPS0 * 2.2 * (1 - 0.02j)
    p = eo.build_problem(d)
    r = dict(p["rwg"])
    r["minusTri"] = r["minusTri"].copy()
    r["minusTri"][5] = 0
    p = dict(p, rwg=r)
    omega, k, _, _ = eo.physics(2.5e9, d.mu, d.eps)
    Z, _ = _gg(p, k, omega)
    Zo = oc.assemble_z(r, p["prepack"], k, omega, d.mu, d.eps)
    assert _rel(Z, Zo) < TOL_Z


def test_asymmetric_near_matrix():
    """A nearMat that is not symmetric disables the t1<=t2 storage; still exact."""
    p = eo.build_problem(small_design("grid"))
    pre = dict(p["prepack"])
    nm = pre["nearMat"].copy()
    i, j = np.nonzero(np.triu(nm, 1))
    nm[i[0], j[0]] = 0
    pre["nearMat"] = np.asfortranarray(nm)
    p = dict(p, prepack=pre)
    d = p["design"]
    omega, k, _, _ = eo.physics(2.2e9, d.mu, d.eps)
    Z, _ = _gg(p, k, omega)
    Zo = oc.assemble_z(p["rwg"], pre, k, omega, d.mu, d.eps)
    assert _rel(Z, Zo) < TOL_Z


def test_rwg_free_vertex_off_its_triangle():
    """A copy of an RWG whose free vertex is moved by 1e-9 of the mesh size
    leaves four distinct free vertices on a triangle: the assembly falls back
    from the nine edge-combination values per triangle pair to the eight
    moments, and stays exact against the oracle."""
    p = eo.build_problem(small_design("grid"))
    r = {k: np.array(v, copy=True) for k, v in p["rwg"].items()}
    e = 5
    for key in ("edge", "plusTri", "minusTri", "plusSign", "minusSign", "rp", "rm", "Ap", "Am", "len", "center",
                "zSign"):
        r[key] = np.asfortranarray(np.concatenate([r[key], r[key][e:e + 1]]))
    r["rp"][-1] += 1e-9 * np.abs(p["V"]).max()
    r["Ne"] = np.int64(r["Ne"] + 1)
    p = dict(p, rwg=r)
    d = p["design"]
    omega, k, _, _ = eo.physics(2.3e9, d.mu, d.eps)
    Z, _ = _gg(p, k, omega)
    Zo = oc.assemble_z(r, p["prepack"], k, omega, d.mu, d.eps)
    assert Z.shape == (r["Ne"], r["Ne"])
    assert _rel(Z, Zo) < TOL_Z


def test_gassemble_matches_oracle_and_reference():
    m = pkg()
    d = small_design("grid")
    p = eo.build_problem(d)
    r = p["rwg"]
    omega, k, _, _ = eo.physics(2.4e9, d.mu, d.eps)
    exc = np.array([p["patchEdge"], p["groundEdge"], d.V0, p["spread"], 0.2])
    Z, V = m.gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(
        p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
        r["Ap"], r["Am"], r["len"], k, omega, d.mu, d.eps, exc)
    Zo = oc.assemble_centroid(p["V"], p["F"], r, 0.2, k, omega, d.mu, d.eps)
    assert _rel(Z, Zo) < 1e-13
    ref_mex = pytest.importorskip("ref_mex")
    Zr, Vr = ref_mex.gassemble(p, k, omega, d.mu, d.eps, 0.2)
    assert _rel(Z, Zr) < 1e-13
    assert np.array_equal(V, Vr)


def test_struct_api_matches_flat_api():
    m = pkg()
    d = small_design("grid")
    p = eo.build_problem(d)
    omega, k, _, _ = eo.physics(2.4e9, d.mu, d.eps)
    rwg = dict(p["rwg"], V=p["V"], F=p["F"])
    pre = dict(p["prepack"])
    pre["self_aSoft"] = pre.pop("self_a")
    exc = dict(patchEdge=p["patchEdge"], groundEdge=p["groundEdge"], V0=1.0, spreadRadius=p["spread"])
    Z1, V1 = m.assemble_ZV_EFIE_RWG_DIFF_GPU_FAST(rwg, pre, k, omega, d.mu, d.eps, exc,
                                                  dict(near_alpha=p["prepack"]["near_alpha"]))
    Z2, V2 = _gg(p, k, omega)
    assert np.array_equal(Z1, Z2) and np.array_equal(V1, V2)
