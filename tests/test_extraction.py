"""Extraction scheme (Dunavant 7-point rule + analytic 1/R extraction on self
and vertex-adjacent pairs).  CPU: the analytic potential integrals against
Duffy-transformed quadrature, and the FP64 oracle's symmetry.  GPU: the
product against the oracle of the same discretisation (|dZ| <= 1e-12 max|Z|),
and sweeps (complex128 LU |dZin|/|Zin| <= 1e-9, mixed <= 1e-6)."""
import importlib

import numpy as np
import pytest

import efie_oracle as eo
import oracle_c as oc
from conftest import small_design, config1_design


@pytest.mark.parametrize("where", ["inside", "outside", "off_plane", "near_edge"])
def test_potential_integrals_match_quadrature(where):
    rng = np.random.default_rng(7)
    a = np.array([[0.0, 0.0, 0.0], [1.2e-3, 0.1e-3, 0.0], [0.3e-3, 0.9e-3, 0.2e-3]])
    for _ in range(5):
        u, v = rng.random(2)
        if u + v > 1:
            u, v = 1 - u, 1 - v
        r = a[0] + u * (a[1] - a[0]) + v * (a[2] - a[0])
        n = np.cross(a[1] - a[0], a[2] - a[0])
        n /= np.linalg.norm(n)
        if where == "outside":
            r = r + (a[1] - a[0]) * 1.3
        elif where == "off_plane":
            r = r + n * rng.uniform(-5e-4, 5e-4)
        elif where == "near_edge":
            r = a[0] + 0.5 * (a[1] - a[0]) + 1e-3 * (r - a[0]) * 0.01
        I0a, Ja = oc.potential_integrals(a, r)
        I0n, Jn = eo.potential_integrals_numeric(a, r, order=300)
        assert abs(I0a - I0n) <= 1e-11 * abs(I0n)
        assert np.abs(Ja - Jn).max() <= 1e-10 * np.abs(Jn).max()


def test_extract_oracle_symmetric_and_finite(small_problem):
    p = small_problem
    d = p["design"]
    omega, k, _, _ = eo.physics(2.5e9, d.mu, d.eps)
    Z = oc.assemble_z_extract(p["V"], p["F"], p["rwg"], k, omega, d.mu, d.eps)
    assert np.all(np.isfinite(Z))
    assert np.abs(Z - Z.T).max() <= 1e-13 * np.abs(Z).max()


def _plan(p, solver):
    m = importlib.import_module("matlab-cuda-efief-vs-cpu_b200")
    r = p["rwg"]
    d = p["design"]
    return m.SweepPlan(p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"],
                       r["rm"], r["Ap"], r["Am"], r["len"], None, d.mu, d.eps, p["patchEdge"], p["groundEdge"], d.V0,
                       p["spread"], d.Z0, opts=m.sweep_opts(solver=solver, scheme="extract"), rule_order=eo.DUNAVANT7)


def _oracle_sweep(p, freqs):
    d = p["design"]
    out = []
    for f in freqs:
        omega, k, _, _ = eo.physics(f, d.mu, d.eps)
        Z = oc.assemble_z_extract(p["V"], p["F"], p["rwg"], k, omega, d.mu, d.eps)
        x = np.linalg.solve(Z, p["b"].astype(complex))
        out.append(eo.zin_s11(eo.port_current(x, p["wP"], p["wG"], p["rwg"]["len"]), d.V0, d.Z0)[0])
    return np.array(out)


@pytest.mark.gpu
@pytest.mark.parametrize("name,design", [("small", lambda: small_design("grid")),
                                         ("config1_1074", lambda: config1_design("grid"))])
@pytest.mark.parametrize("solver,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_extract_sweep_matches_oracle(name, design, solver, tol):
    d = design()
    p = eo.build_problem(d)
    freqs = d.freqs[[0, -1]]
    plan = _plan(p, solver)
    Zin, _, I = plan.run(freqs, return_currents=True)
    Zo = _oracle_sweep(p, freqs)
    assert (np.abs(Zin - Zo) / np.abs(Zo)).max() <= tol
    # the currents solve the oracle's Z to the refinement tolerance
    omega, k, _, _ = eo.physics(freqs[0], d.mu, d.eps)
    Z = oc.assemble_z_extract(p["V"], p["F"], p["rwg"], k, omega, d.mu, d.eps)
    assert np.linalg.norm(p["b"] - Z @ I[:, 0]) / np.linalg.norm(p["b"]) <= 1e-9
    plan.close()
