"""efie_precompute + efie_precompute_pack on the GPU (efie_precompute.m:1-97,
efie_precompute_pack.m:1-59) against the numpy restatement of the oracle and
the host producer: nearMat bit-exact, every floating-point array within
1e-15 relative (by construction the device rounds every operation as the
host does, so the arrays are expected to be identical).  A plan whose prepack
is computed on the device sweeps bit-identically to one created from the host
prepack."""
import numpy as np
import pytest

import efie_oracle as eo
from conftest import pkg, small_design, config1_design

pytestmark = pytest.mark.gpu

FLOAT_FIELDS = ("r_reg", "w_reg", "self_r", "self_w", "self_a", "near_r", "near_w", "aeqTri")


@pytest.mark.parametrize("opts", [eo.DEFAULT_OPTS_GPU, eo.DEFAULT_OPTS_ACCURATE,
                                  dict(quad_order=-7, near_sing_eps=2.0, self_subdiv=3, near_subdiv=0,
                                       near_order=1, self_alpha=0.3, near_alpha=0.1)],
                         ids=["gpu_set", "accurate_set", "dunavant_deep"])
@pytest.mark.parametrize("design", ["small_reference_order", "config1"])
def test_device_prepack_matches_oracle_and_host(opts, design):
    m = pkg()
    d = small_design("reference") if design == "small_reference_order" else config1_design("grid")
    V, F = eo.make_patch_with_ground_mesh(d.Lp, d.Wp, d.Lg, d.Wg, d.h, d.Np_x, d.Np_y, d.Ng_x, d.Ng_y,
                                          vertex_order=d.vertex_order)
    ref = eo.efie_precompute_pack(V, F, opts)
    gpu = m.efie_precompute_pack_gpu({"V": V, "F": F}, opts)
    host = m.efie_precompute_pack({"V": V, "F": F}, opts)
    assert np.array_equal(gpu["nearMat"], ref["nearMat"])
    assert gpu["nearMat"].dtype == np.uint8
    for f in FLOAT_FIELDS:
        a, b = np.asarray(gpu[f]).reshape(-1, order="F"), np.asarray(ref[f]).reshape(-1, order="F")
        assert a.shape == b.shape, f
        assert np.abs(a - b).max() <= 1e-15 * np.abs(b).max(), f
        assert np.array_equal(np.asarray(gpu[f]), np.asarray(host[f])), f
    assert gpu["near_alpha"] == ref["near_alpha"] and gpu["self_alpha"] == ref["self_alpha"]


def test_plan_from_device_prepack_sweeps_like_the_host_prepack():
    m = pkg()
    d = config1_design("grid")
    p = eo.build_problem(d)
    r = p["rwg"]
    args = [p["V"], p["F"], r["edge"], r["plusTri"], r["minusTri"], r["plusSign"], r["minusSign"], r["rp"], r["rm"],
            r["Ap"], r["Am"], r["len"]]
    tail = [d.mu, d.eps, p["patchEdge"], p["groundEdge"], d.V0, p["spread"], d.Z0]
    freqs = d.freqs[[0, 4, 9]]
    out = []
    for pre, popts in ((p["prepack"], None), (None, d.opts)):
        for solver in ("fp64", "mixed"):
            plan = m.SweepPlan(*args, pre, *tail, opts=m.sweep_opts(solver=solver), precompute=popts)
            out.append(plan.run(freqs, return_currents=True))
            plan.close()
    for (a, b) in ((out[0], out[2]), (out[1], out[3])):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])
    Zo, _ = eo.solve_sweep(p, freqs, assemble=__import__("oracle_c").assemble_z)
    assert (np.abs(out[3][0] - Zo) / np.abs(Zo)).max() <= 1e-6
