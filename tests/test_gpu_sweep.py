"""GPU parity of the frequency sweeps (assemble + solve + Zin/S11) against the
FP64 oracle (C assembly + LAPACK solve) and the reference's own CUDA sweep.
Tolerances: complex128 LU path |dZin|/|Zin| <= 1e-9; mixed path (complex64
tensor-core LU + FP64 refinement to 1e-10) |dZin|/|Zin| <= 1e-6."""
import numpy as np
import pytest

import efie_oracle as eo
import oracle_c as oc
from conftest import pkg, small_design, config1_design

pytestmark = pytest.mark.gpu


def _sweep(p, freqs, solver, **kw):
    m = pkg()
    r = p["rwg"]
    d = p["design"]
    st = {}
    out = m.patch_sweep_fastquad_cuda(
        p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
        r["Ap"], r["Am"], r["len"], p["prepack"], np.asarray(freqs, np.float64), d.mu, d.eps, p["patchEdge"],
        p["groundEdge"], d.V0, p["spread"], d.Z0, opts=m.sweep_opts(solver=solver, **kw), stats=st)
    return out[0], out[1], st


def _oracle(p, freqs):
    return eo.solve_sweep(p, freqs, assemble=oc.assemble_z)


@pytest.mark.parametrize("name,design", [("small", lambda: small_design("grid")),
                                         ("reference_sweep_538", eo.reference_sweep_design),
                                         ("config1_1074", lambda: config1_design("grid"))])
@pytest.mark.parametrize("solver,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_sweep_matches_oracle(name, design, solver, tol):
    d = design()
    p = eo.build_problem(d)
    freqs = d.freqs[[0, len(d.freqs) // 2, -1]]
    Zin, S11, st = _sweep(p, freqs, solver)
    Zo, So = _oracle(p, freqs)
    err = np.abs(Zin - Zo) / np.abs(Zo)
    assert err.max() <= tol, err
    assert np.abs(S11 - So).max() <= 10 * tol
    if solver == "mixed":
        assert st["max_relres"] <= 1e-10 and st["n_fp64_fallback"] == 0


def test_sweep_matches_reference_cuda():
    ref_mex = pytest.importorskip("ref_mex")
    d = eo.reference_sweep_design()
    p = eo.build_problem(d)
    freqs = d.freqs[::10]
    Zr, Sr = ref_mex.patch_sweep_fastquad(p, freqs)
    for solver, tol in (("fp64", 1e-9), ("mixed", 1e-6)):
        Zin, S11, _ = _sweep(p, freqs, solver)
        assert (np.abs(Zin - Zr) / np.abs(Zr)).max() <= tol


def test_refinement_fallback_to_fp64():
    """A refinement that cannot reach its target re-solves with the complex128 LU."""
    d = small_design("grid")
    p = eo.build_problem(d)
    freqs = d.freqs
    Zin, _, st = _sweep(p, freqs, "mixed", refine_tol=1e-30, refine_max_iter=2)
    assert st["n_fp64_fallback"] == len(freqs)
    Zo, _ = _oracle(p, freqs)
    assert (np.abs(Zin - Zo) / np.abs(Zo)).max() <= 1e-9


def test_centroid_sweep_matches_reference():
    m = pkg()
    d = small_design("grid")
    p = eo.build_problem(d)
    r = p["rwg"]
    Zin, S11 = m.patch_sweep_cuda(p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"],
                                  r["minusSign"], r["rp"], r["rm"], r["Ap"], r["Am"], r["len"], d.freqs, d.mu,
                                  d.eps, np.int32(p["patchEdge"]), np.int32(p["groundEdge"]), d.V0, p["spread"],
                                  d.Z0)
    # oracle: centroid Z, LAPACK solve, edge-difference port
    Zo = []
    for f in d.freqs:
        omega, k, _, _ = eo.physics(f, d.mu, d.eps)
        Z = oc.assemble_centroid(p["V"], p["F"], r, 0.2, k, omega, d.mu, d.eps)
        x = np.linalg.solve(Z, p["b"].astype(complex))
        Zo.append(d.V0 / (x[p["patchEdge"] - 1] - x[p["groundEdge"] - 1]))
    Zo = np.array(Zo)
    assert (np.abs(Zin - Zo) / np.abs(Zo)).max() <= 1e-6
    ref_mex = pytest.importorskip("ref_mex")
    Zr, Sr = ref_mex.patch_sweep_cuda(p, d.freqs)
    assert (np.abs(Zin - Zr) / np.abs(Zr)).max() <= 1e-6


def test_plan_reuse_and_currents():
    m = pkg()
    d = small_design("grid")
    p = eo.build_problem(d)
    r = p["rwg"]
    plan = m.SweepPlan(p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"],
                       r["rp"], r["rm"], r["Ap"], r["Am"], r["len"], p["prepack"], d.mu, d.eps, p["patchEdge"],
                       p["groundEdge"], d.V0, p["spread"], d.Z0)
    a = plan.run(d.freqs, return_currents=True)
    b = plan.run(d.freqs, return_currents=True)
    assert np.array_equal(a[0], b[0])
    omega, k, _, _ = eo.physics(d.freqs[0], d.mu, d.eps)
    Z = oc.assemble_z(r, p["prepack"], k, omega, d.mu, d.eps)
    x = a[2][:, 0]
    assert np.linalg.norm(p["b"] - Z @ x) / np.linalg.norm(p["b"]) < 1e-9
    plan.close()


@pytest.mark.parametrize("spacing", ["even", "uneven"])
def test_multi_frequency_assembly_matches_oracle(spacing):
    """Equally spaced frequencies of a batch share one regular-pair launch
    (e^{-jk_f R} by recurrence in f); unevenly spaced ones are assembled one by
    one.  The currents solve the oracle's Z of each frequency to 1e-9."""
    m = pkg()
    d = config1_design("grid")
    p = eo.build_problem(d)
    r = p["rwg"]
    freqs = np.linspace(d.freqs[0], d.freqs[-1], 4)
    if spacing == "uneven":
        freqs[1] *= 1.001
    plan = m.SweepPlan(p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"],
                       r["rp"], r["rm"], r["Ap"], r["Am"], r["len"], p["prepack"], d.mu, d.eps, p["patchEdge"],
                       p["groundEdge"], d.V0, p["spread"], d.Z0, opts=m.sweep_opts(batch=4))
    _, _, I = plan.run(freqs, return_currents=True)
    plan.close()
    for j, f in enumerate(freqs):
        omega, k, _, _ = eo.physics(f, d.mu, d.eps)
        Z = oc.assemble_z(r, p["prepack"], k, omega, d.mu, d.eps)
        x = I[:, j]
        assert np.linalg.norm(p["b"] - Z @ x) / np.linalg.norm(p["b"]) < 1e-9


@pytest.mark.parametrize("lu_nb", [128, 256, 512])
def test_panel_widths_match_oracle(lu_nb):
    """Every outer panel width of the two-level LU (the K of the tensor-core
    trailing updates) reaches the refinement target and the oracle's Zin."""
    d = config1_design("grid")
    p = eo.build_problem(d)
    freqs = d.freqs[:4]
    Zb, _, st = _sweep(p, freqs, "mixed", lu_nb=lu_nb)
    Zo, _ = _oracle(p, freqs)
    assert (np.abs(Zb - Zo) / np.abs(Zo)).max() <= 1e-6
    assert st["n_fp64_fallback"] == 0 and st["max_relres"] <= 1e-10


@pytest.mark.parametrize("batch", [1, 2, 4])
def test_batched_sweep_matches_unbatched(batch):
    """Frequencies solved together (ragged last batch) give the same Zin."""
    d = config1_design("grid")
    p = eo.build_problem(d)
    freqs = d.freqs[:5]
    Zb, Sb, st = _sweep(p, freqs, "mixed", batch=batch)
    Zo, _ = _oracle(p, freqs)
    assert (np.abs(Zb - Zo) / np.abs(Zo)).max() <= 1e-6
    assert st["n_fp64_fallback"] == 0 and st["max_relres"] <= 1e-10


def test_gmres_converges_where_classical_refinement_stalls():
    """cfg2 (Ne 6968) near 2.4-2.5 GHz, where u32 * cond(Z) comes close to 1:
    flexible GMRES with the complex64 LU converges to 1e-10 without a
    complex128 fallback, in no more steps than classical refinement with the
    same LU (which may stall there and fall back), and matches the complex128
    LU to 1e-6."""
    d = eo.Design(Lp=30e-3, Wp=38e-3, Lg=60e-3, Wg=60e-3, h=1.6e-3, Np_x=32, Np_y=24, Ng_x=40, Ng_y=40,
                  feed=(0.0, -7e-3), vertex_order="grid", opts=dict(eo.DEFAULT_OPTS_GPU),
                  freqs=np.linspace(2e9, 3e9, 101)[40:48])
    p = eo.build_problem(d)
    Z64, _, _ = _sweep(p, d.freqs, "fp64")
    Zc, _, stc = _sweep(p, d.freqs, "mixed", refine="classical")
    Zg, _, stg = _sweep(p, d.freqs, "mixed", refine="gmres")
    assert stg["n_fp64_fallback"] == 0 and stg["max_relres"] <= 1e-10
    assert stc["n_fp64_fallback"] > 0 or stg["refine_iters_max"] <= stc["refine_iters_max"]
    assert (np.abs(Zg - Z64) / np.abs(Z64)).max() <= 1e-6
    assert (np.abs(Zc - Z64) / np.abs(Z64)).max() <= 1e-6


def test_graph_replay_matches_eager_launches():
    """The mixed factorization replayed from a captured CUDA graph (timing off)
    gives bit-identical results to eager launches (timing on), and later
    batches of the same plan replay the graph (the reversed sweep within the
    refinement tolerance)."""
    m = pkg()
    d = config1_design("grid")
    p = eo.build_problem(d)
    r = p["rwg"]
    args = [p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
            r["Ap"], r["Am"], r["len"], p["prepack"], d.mu, d.eps, p["patchEdge"], p["groundEdge"], d.V0, p["spread"],
            d.Z0]
    freqs = d.freqs
    import torch
    s = torch.cuda.Stream()
    nat = __import__(m.__name__ + "._native", fromlist=["x"])
    nat.check(nat.lib().efie_ctx_set_stream(nat.context(), s.cuda_stream))
    try:
        eager = m.SweepPlan(*args, opts=m.sweep_opts(timing=True, batch=4))
        Ze, Se = eager.run(freqs)
        eager.close()
        graph = m.SweepPlan(*args, opts=m.sweep_opts(timing=False, batch=4))
        Zg, Sg = graph.run(freqs)          # 3 batches: capture on the first, replay on the others
        Zg2, _ = graph.run(freqs[::-1])
        graph.close()
    finally:
        nat.check(nat.lib().efie_ctx_set_stream(nat.context(), None))
    assert np.array_equal(Zg, Ze) and np.array_equal(Sg, Se)
    # in reverse order the frequencies share their regular-pair launches with
    # other neighbours (e^{-jk_f R} by recurrence from the group's first
    # frequency): Z moves in its last bits, Zin within the GMRES tolerance
    assert np.abs(Zg2 - Zg[::-1]).max() <= 1e-8 * np.abs(Zg).max()


def test_coarse_to_fine_batches_with_interpolated_guesses():
    """Several batches of the mixed solver run coarse to fine (sorted
    positions by residue, van der Corput order) and start GMRES from the
    interpolation of solved neighbours.  Unsorted input frequencies come back
    in their own order, currents included, and match the same sweep with
    every refinement started from zero and the oracle."""
    m = pkg()
    nat = __import__(m.__name__ + "._native", fromlist=["x"])
    d = config1_design("grid")
    p = eo.build_problem(d)
    r = p["rwg"]
    args = [p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
            r["Ap"], r["Am"], r["len"], p["prepack"], d.mu, d.eps, p["patchEdge"], p["groundEdge"], d.V0, p["spread"],
            d.Z0]
    freqs = np.linspace(d.freqs[0], d.freqs[-1], 13)
    perm = np.random.default_rng(5).permutation(len(freqs))
    plan = m.SweepPlan(*args, opts=m.sweep_opts(batch=3))
    Zw, Sw, Iw = plan.run(freqs[perm], return_currents=True)
    nat.lib().efie_debug_disable_warm_start(1)
    try:
        Zc, Sc, Ic = plan.run(freqs, return_currents=True)
    finally:
        nat.lib().efie_debug_disable_warm_start(0)
    plan.close()
    assert (np.abs(Zw - Zc[perm]) / np.abs(Zc[perm])).max() <= 1e-7
    Zo, _ = _oracle(p, freqs[perm])
    assert (np.abs(Zw - Zo) / np.abs(Zo)).max() <= 1e-6
    for j in (0, 7, 12):
        omega, k, _, _ = eo.physics(freqs[perm[j]], d.mu, d.eps)
        Z = oc.assemble_z(r, p["prepack"], k, omega, d.mu, d.eps)
        assert np.linalg.norm(p["b"] - Z @ Iw[:, j]) / np.linalg.norm(p["b"]) < 1e-9


def test_asymmetric_near_matrix_sweep_in_batches():
    """A nearMat that is not symmetric keeps the general gather, the general
    LU and the full GMRES products; several warm-started batches still match
    the oracle."""
    p = eo.build_problem(small_design("grid"))
    pre = dict(p["prepack"])
    nm = pre["nearMat"].copy()
    i, j = np.nonzero(np.triu(nm, 1))
    nm[i[0], j[0]] = 0
    pre["nearMat"] = np.asfortranarray(nm)
    p = dict(p, prepack=pre)
    d = p["design"]
    freqs = np.linspace(d.freqs[0], d.freqs[-1], 7)
    Zin, _, st = _sweep(p, freqs, "mixed", batch=2)
    Zo, _ = _oracle(p, freqs)
    assert (np.abs(Zin - Zo) / np.abs(Zo)).max() <= 1e-6
    assert st["n_fp64_fallback"] == 0 and st["max_relres"] <= 1e-10


def test_repeated_frequencies_in_warm_started_sweep():
    """Repeated frequencies (the interpolation then takes the nearest solved
    one) give the same Zin as their first occurrence."""
    d = config1_design("grid")
    p = eo.build_problem(d)
    f = np.linspace(d.freqs[0], d.freqs[-1], 5)
    freqs = np.array([f[0], f[2], f[2], f[4], f[1], f[1], f[3]])
    Zin, _, st = _sweep(p, freqs, "mixed", batch=2)
    Zo, _ = _oracle(p, freqs)
    assert (np.abs(Zin - Zo) / np.abs(Zo)).max() <= 1e-6
    assert abs(Zin[1] - Zin[2]) <= 1e-7 * abs(Zin[1]) and abs(Zin[4] - Zin[5]) <= 1e-7 * abs(Zin[4])
    assert st["n_fp64_fallback"] == 0


@pytest.mark.parametrize("group", [2, 4])
def test_shared_factors_match_every_frequency_factored(group):
    """With shared factors only the first of each group of coarse-to-fine
    batches is factored; the other frequencies refine with the complex64
    factors of their nearest factored neighbour.  GMRES reaches the same
    residual target, so Zin agrees with the sweep that factors every
    frequency and with the oracle, every solved current meets the residual
    target, and the stats count the frequencies that shared factors."""
    m = pkg()
    d = config1_design("grid")
    p = eo.build_problem(d)
    r = p["rwg"]
    args = [p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
            r["Ap"], r["Am"], r["len"], p["prepack"], d.mu, d.eps, p["patchEdge"], p["groundEdge"], d.V0, p["spread"],
            d.Z0]
    freqs = np.linspace(d.freqs[0], d.freqs[-1], 17)
    full = m.SweepPlan(*args, opts=m.sweep_opts(share_factors=1, nfreq_hint=len(freqs)))
    Zf, _ = full.run(freqs)
    assert full.stats["n_shared_factors"] == 0
    full.close()
    plan = m.SweepPlan(*args, opts=m.sweep_opts(share_factors=group, nfreq_hint=len(freqs)))
    Zs, _, Is = plan.run(freqs, return_currents=True)
    st = plan.stats
    plan.close()
    # `group` balanced batches, one group: every frequency outside the first
    # batch (sorted positions 0, g, 2g, ...) shares its factors
    assert st["n_shared_factors"] == len(freqs) - -(-len(freqs) // group)
    assert st["n_fp64_fallback"] == 0
    assert st["max_relres"] <= 1e-10
    assert (np.abs(Zs - Zf) / np.abs(Zf)).max() <= 1e-7
    Zo, _ = _oracle(p, freqs)
    assert (np.abs(Zs - Zo) / np.abs(Zo)).max() <= 1e-6
    for j in (1, 8, 15):
        omega, k, _, _ = eo.physics(freqs[j], d.mu, d.eps)
        Z = oc.assemble_z(r, p["prepack"], k, omega, d.mu, d.eps)
        assert np.linalg.norm(p["b"] - Z @ Is[:, j]) / np.linalg.norm(p["b"]) < 1e-9
