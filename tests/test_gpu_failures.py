"""Failure paths of the sweeps, made on the host (no GPU fault, no hang).

* A Z that is exactly singular -- one RWG whose edge length is zero, so its
  row and column of Z are zero -- ends the sweep with ``efie:singular`` on both
  solvers.  The reference never reads cuSOLVER's ``info``
  (patch_sweep_fastquad_cuda.cu:770) and returns Inf/NaN there instead.
* A bounded device wait that runs out: the test hook makes every wait of the
  triangular solves target a count that no block publishes, so each wait gives
  up after a short limit, records a timeout and returns.  The frequencies are
  then re-solved by the complex128 LU and match the oracle; with the hook off
  the same sweep needs no fallback.
* Very low frequencies (the EFIE's low-frequency breakdown, cond(Z) growing as
  1/f^2): where the complex64 factors no longer precondition GMRES to the
  target, the sweep retries the general LU and then falls back to the
  complex128 LU, without a forced tolerance, and still matches the oracle.
"""
import numpy as np
import pytest

import efie_oracle as eo
import oracle_c as oc
from conftest import pkg, small_design, config1_design

pytestmark = pytest.mark.gpu


def _sweep(p, freqs, solver="mixed", rwg=None, **kw):
    m = pkg()
    r = rwg or p["rwg"]
    d = p["design"]
    st = {}
    Zin, S11 = m.patch_sweep_fastquad_cuda(
        p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
        r["Ap"], r["Am"], r["len"], p["prepack"], np.asarray(freqs, np.float64), d.mu, d.eps, p["patchEdge"],
        p["groundEdge"], d.V0, p["spread"], d.Z0, opts=m.sweep_opts(solver=solver, **kw), stats=st)
    return Zin, st


@pytest.mark.parametrize("solver", ["mixed", "fp64"])
def test_zero_rwg_makes_the_sweep_singular(solver):
    m = pkg()
    p = eo.build_problem(small_design("grid"))
    r = dict(p["rwg"])
    j = next(e for e in range(r["Ne"]) if e + 1 not in (p["patchEdge"], p["groundEdge"]))
    r["len"] = r["len"].copy()
    r["len"][j] = 0.0
    with pytest.raises(m.MexError) as ei:
        _sweep(p, p["design"].freqs[:2], solver, rwg=r)
    assert ei.value.identifier == "efie:singular"
    assert "frequency index 1" in str(ei.value)


def test_wait_timeout_falls_back_to_the_complex128_lu():
    m = pkg()
    nat = __import__(m.__name__ + "._native", fromlist=["x"])
    p = eo.build_problem(config1_design("grid"))
    freqs = p["design"].freqs[[0, 5, 10]]
    nat.check(nat.lib().efie_debug_set_wait_test(1, 1 << 12))
    try:
        Zt, st = _sweep(p, freqs)
    finally:
        nat.check(nat.lib().efie_debug_set_wait_test(0, 0))
    assert st["n_wait_timeouts"] == len(freqs) and st["n_fp64_fallback"] == len(freqs)
    Zo, _ = eo.solve_sweep(p, freqs, assemble=oc.assemble_z)
    assert (np.abs(Zt - Zo) / np.abs(Zo)).max() <= 1e-9
    Zn, st2 = _sweep(p, freqs)
    assert st2["n_wait_timeouts"] == 0 and st2["n_fp64_fallback"] == 0
    assert (np.abs(Zn - Zo) / np.abs(Zo)).max() <= 1e-6


def test_low_frequency_breakdown_falls_back_without_forced_tolerance():
    p = eo.build_problem(config1_design("grid"))
    freqs = np.array([2.0e6, 2.0e9])
    Zin, st = _sweep(p, freqs)
    assert st["n_fp64_fallback"] >= 1
    Zo, _ = eo.solve_sweep(p, freqs, assemble=oc.assemble_z)
    assert (np.abs(Zin - Zo) / np.abs(Zo)).max() <= 1e-6
