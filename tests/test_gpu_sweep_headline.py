"""Zin parity on the workloads the throughput is quoted on.

cfg2 (patch 38x30 mm as 32x24 over a 60x60 mm ground as 40x40, Ne 6968,
101 points over 2-3 GHz) runs the default mixed solver exactly as the bench
does: coarse-to-fine batches of up to 32 frequencies, GMRES warm-started from
interpolated neighbours, 512-column outer panels of the symmetric tensor-core
LU, multi-frequency regular-pair assembly.  Its Zin is compared with

* the package's plain FP64 GPU path (complex128 assembly + cuSOLVER
  Zgetrf/Zgetrs, the reference's solve, patch_sweep_fastquad_cuda.cu:765-799)
  on all 101 points, and
* the CPU oracle (C restatement of CPU_FAST + LAPACK, the reference's CPU path
  main_patch_efie_rwg_fast.m:116-133) on five points, including the one
  furthest from the FP64 path.

cfg5 (patch 40x32 mm at 0.5 mm over a 90x90 mm ground as 40x40, Ne 19936)
runs the mixed solver on three of its 51 points against the FP64 GPU path.
Tolerance: |dZin|/|Zin| <= 1e-6 (mixed), <= 1e-9 (FP64 path vs the oracle).
"""
import numpy as np
import pytest

import efie_oracle as eo
import oracle_c as oc
from conftest import pkg

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-6
TOL_FP64 = 1e-9


def _cfg2():
    return eo.Design(Lp=30e-3, Wp=38e-3, Lg=60e-3, Wg=60e-3, h=1.6e-3, Np_x=32, Np_y=24, Ng_x=40, Ng_y=40,
                     feed=(0.0, -7e-3), vertex_order="grid", opts=dict(eo.DEFAULT_OPTS_GPU),
                     freqs=np.linspace(2e9, 3e9, 101))


def _sweep(p, freqs, **kw):
    m = pkg()
    r = p["rwg"]
    d = p["design"]
    st = {}
    Zin, S11 = m.patch_sweep_fastquad_cuda(
        p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
        r["Ap"], r["Am"], r["len"], p["prepack"], np.asarray(freqs, np.float64), d.mu, d.eps, p["patchEdge"],
        p["groundEdge"], d.V0, p["spread"], d.Z0, opts=m.sweep_opts(**kw), stats=st)
    return Zin, S11, st


@pytest.fixture(scope="module")
def cfg2_problem():
    return eo.build_problem(_cfg2())


def test_cfg2_mixed_sweep_matches_fp64_path_and_cpu_oracle(cfg2_problem):
    p = cfg2_problem
    freqs = p["design"].freqs
    Zm, Sm, st = _sweep(p, freqs)                  # the default: mixed solver, automatic batches
    Z64, S64, st64 = _sweep(p, freqs, solver="fp64")
    assert st["n_fp64_fallback"] == 0 and st["max_relres"] <= 1e-10
    err = np.abs(Zm - Z64) / np.abs(Z64)
    assert err.max() <= TOL_MIXED, (err.max(), int(err.argmax()))
    assert np.abs(Sm - S64).max() <= 10 * TOL_MIXED
    idx = sorted({0, 37, 62, 100, int(err.argmax())})
    Zo, _ = eo.solve_sweep(p, freqs[idx], assemble=oc.assemble_z)
    e_mixed = np.abs(Zm[idx] - Zo) / np.abs(Zo)
    e_fp64 = np.abs(Z64[idx] - Zo) / np.abs(Zo)
    assert e_mixed.max() <= TOL_MIXED, e_mixed
    assert e_fp64.max() <= TOL_FP64, e_fp64


def test_cfg5_mixed_points_match_fp64_path():
    m = pkg()
    V, F, _, _ = m.make_patch_with_ground_mesh(32e-3, 40e-3, 90e-3, 90e-3, 1.6e-3, 80, 64, 40, 40,
                                               vertex_order="grid")
    rwg = m.build_rwg_interior({"V": V, "F": F})
    assert rwg["Ne"] == 19936
    pe = m.pick_port_edge_by_point_and_layer(rwg, (0.0, -7e-3, +0.8e-3), +1)
    ge = m.pick_port_edge_by_point_and_layer(rwg, (0.0, -7e-3, -0.8e-3), -1)
    pre = m.efie_precompute_pack({"V": V, "F": F}, eo.DEFAULT_OPTS_GPU)
    d = eo.Design(Lp=32e-3, Wp=40e-3, Lg=90e-3, Wg=90e-3, h=1.6e-3, Np_x=80, Np_y=64, Ng_x=40, Ng_y=40)
    p = dict(V=V, F=F, rwg=rwg, patchEdge=pe, groundEdge=ge, spread=1.5 * float(np.mean(rwg["len"])),
             prepack=pre, design=d)
    freqs = np.linspace(2e9, 3e9, 51)[[0, 25, 50]]
    Zm, _, st = _sweep(p, freqs)
    Z64, _, _ = _sweep(p, freqs, solver="fp64")
    assert st["n_fp64_fallback"] == 0 and st["max_relres"] <= 1e-10
    err = np.abs(Zm - Z64) / np.abs(Z64)
    assert err.max() <= TOL_MIXED, err
