"""CPU tests of the oracle: invariants the reference implies, agreement of
the two independent restatements, and the golden vectors made by the
reference's own CUDA code (tests/golden)."""
import os

import numpy as np
import pytest

import efie_oracle as eo
import oracle_c as oc
from conftest import small_design, config1_design

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("order", [1, 2, 4, eo.DUNAVANT7])
def test_quad_weights_sum_half(order):
    qp, qw = eo.tri_quad_rule(order)
    assert abs(qw.sum() - 0.5) < 1e-14                       # tri_quad_rule.m:11,21


def test_dunavant7_exact_to_degree5():
    qp, qw = eo.dunavant7()
    # exact integral over the reference triangle of u^a v^b = a! b! / (a+b+2)!
    from math import factorial
    for a in range(6):
        for b in range(6 - a):
            exact = factorial(a) * factorial(b) / factorial(a + b + 2)
            approx = np.sum(qw * qp[:, 0] ** a * qp[:, 1] ** b)
            assert abs(approx - exact) < 1e-15


def test_rwg_counts_and_orientation():
    for (nx, ny) in [(4, 3), (12, 10), (8, 6)]:
        for order in ("grid", "reference"):
            V, F = eo.make_patch_with_ground_mesh(1e-2, 1.2e-2, 3e-2, 3e-2, 1e-3, nx, ny, 6, 6, order)
            rwg = eo.build_rwg_interior(V, F)
            expect = (3 * nx * ny - nx - ny) + (3 * 36 - 12)
            assert rwg["Ne"] == expect
            assert np.all(rwg["plusTri"] < rwg["minusTri"])     # first incidence = lower triangle
            assert np.all(rwg["plusSign"] == -rwg["minusSign"])  # consistently oriented mesh
            assert np.all(np.diff(rwg["edge"][:, 0].astype(np.int64) * 10**6 + rwg["edge"][:, 1]) > 0)


def test_reference_vertex_order_scrambles_non_square_grids():
    V, F = eo.make_patch_with_ground_mesh(1e-2, 1.2e-2, 3e-2, 3e-2, 1e-3, 4, 3, 6, 6, "reference")
    Vg, Fg = eo.make_patch_with_ground_mesh(1e-2, 1.2e-2, 3e-2, 3e-2, 1e-3, 4, 3, 6, 6, "grid")
    a = eo.build_rwg_interior(V, F)
    b = eo.build_rwg_interior(Vg, Fg)
    assert np.array_equal(a["edge"], b["edge"])          # same topology
    assert a["len"].max() > 1.5 * b["len"].max()          # stretched triangles


def test_rhs_sums_to_zero(small_problem):
    assert abs(small_problem["b"].sum()) < 1e-15


def test_reference_design_size(ref_problem):
    assert ref_problem["rwg"]["Ne"] == 538                    # README: 538 RWG
    assert ref_problem["F"].shape[0] == 384


def test_c_oracle_matches_numpy_oracle(small_problem):
    p = small_problem
    d = p["design"]
    omega, k, _, _ = eo.physics(2.5e9, d.mu, d.eps)
    Zn = eo.assemble_Z_ref(p["rwg"], p["prepack"], k, omega, d.mu, d.eps)
    Zc = oc.assemble_z(p["rwg"], p["prepack"], k, omega, d.mu, d.eps)
    assert np.abs(Zc - Zn).max() / np.abs(Zn).max() < 1e-13
    assert np.abs(Zc - Zc.T).max() / np.abs(Zc).max() < 1e-13  # complex symmetric


def test_c_oracle_accurate_option_set():
    p = eo.build_problem(small_design(opts=eo.DEFAULT_OPTS_ACCURATE, npx=3, npy=2, ngx=4, ngy=4))
    d = p["design"]
    omega, k, _, _ = eo.physics(2.0e9, d.mu, d.eps)
    Zn = eo.assemble_Z_ref(p["rwg"], p["prepack"], k, omega, d.mu, d.eps)
    Zc = oc.assemble_z(p["rwg"], p["prepack"], k, omega, d.mu, d.eps)
    assert np.abs(Zc - Zn).max() / np.abs(Zn).max() < 1e-13


def test_centroid_oracle_symmetric(small_problem):
    p = small_problem
    d = p["design"]
    omega, k, _, _ = eo.physics(2.5e9, d.mu, d.eps)
    Z = oc.assemble_centroid(p["V"], p["F"], p["rwg"], 0.2, k, omega, d.mu, d.eps)
    assert np.abs(Z - Z.T).max() / np.abs(Z).max() < 1e-14


def _golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip("golden fixture %s not generated yet" % name)
    return np.load(path, allow_pickle=False)


@pytest.mark.parametrize("case", ["small_grid_gpu", "small_ref_gpu", "small_grid_accurate"])
def test_oracle_matches_reference_golden_Z(case):
    g = _golden("ggassemble_%s.npz" % case)
    p = eo.build_problem(_design_from_case(case))
    d = p["design"]
    Zc = oc.assemble_z(p["rwg"], p["prepack"], complex(g["k"]), float(g["omega"]), d.mu, d.eps)
    rel = np.abs(Zc - g["Z"]).max() / np.abs(g["Z"]).max()
    assert rel < 1e-12, rel
    b, _, _ = eo.rhs_edge_strip_diff_gaussian(p["V"], p["rwg"]["edge"], p["patchEdge"], p["groundEdge"], d.V0,
                                              p["spread"])
    assert np.abs(b - g["Vrhs"].real).max() < 1e-15


def test_oracle_matches_reference_golden_centroid():
    g = _golden("gassemble_small_grid.npz")
    p = eo.build_problem(_design_from_case("small_grid_gpu"))
    d = p["design"]
    Zc = oc.assemble_centroid(p["V"], p["F"], p["rwg"], 0.2, complex(g["k"]), float(g["omega"]), d.mu, d.eps)
    assert np.abs(Zc - g["Z"]).max() / np.abs(g["Z"]).max() < 1e-13


def test_oracle_matches_reference_golden_sweep():
    g = _golden("patch_sweep_fastquad_refdesign.npz")
    p = eo.build_problem(eo.reference_sweep_design())
    idx = g["freq_idx"]
    Zin, S11 = eo.solve_sweep(p, eo.reference_sweep_design().freqs[idx], assemble=oc.assemble_z)
    assert np.abs(Zin - g["Zin"][idx]).max() / np.abs(g["Zin"][idx]).max() < 1e-9
    assert np.abs(S11 - g["S11"][idx]).max() < 1e-9


def _design_from_case(case):
    if case == "small_grid_gpu":
        return small_design("grid")
    if case == "small_ref_gpu":
        return small_design("reference")
    if case == "small_grid_accurate":
        return small_design("grid", opts=eo.DEFAULT_OPTS_ACCURATE, npx=3, npy=2, ngx=4, ngy=4)
    raise ValueError(case)
