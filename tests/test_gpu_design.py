"""The two-plate mesh, RWG numbering and port edges built on the GPU
(make_patch_with_ground_mesh.m, build_rwg_interior.m,
pick_port_edge_by_point_and_layer.m) against the numpy restatement of the
oracle: every integer output bit-exact (RWG order, plus/minus triangles,
signs, port edges) and every floating-point output identical."""
import numpy as np
import pytest

import efie_oracle as eo
from conftest import pkg

pytestmark = pytest.mark.gpu

CASES = [
    # (Lp, Wp, Lg, Wg, h, Npx, Npy, Ngx, Ngy, feed, vertex_order)
    (12e-3, 16e-3, 30e-3, 30e-3, 1.6e-3, 4, 3, 6, 6, (0.0, -2e-3), "grid"),
    (12e-3, 16e-3, 30e-3, 30e-3, 1.6e-3, 4, 3, 6, 6, (0.0, -2e-3), "reference"),
    (30e-3, 38e-3, 60e-3, 60e-3, 1.6e-3, 12, 10, 16, 16, (0.0, -7e-3), "grid"),
    (20.1e-3, 20.1e-3, 0.2, 0.2, 1.59e-3, 8, 6, 12, 12, (-20.1e-3 / 2 + 1e-3, -20.1e-3 / 2 + 13.2e-3), "reference"),
    (30e-3, 38e-3, 60e-3, 60e-3, 1.6e-3, 32, 24, 40, 40, (0.0, -7e-3), "grid"),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "%dx%d_%dx%d_%s" % (c[5], c[6], c[7], c[8], c[10]))
def test_device_design_matches_oracle(case):
    m = pkg()
    Lp, Wp, Lg, Wg, h, npx, npy, ngx, ngy, feed, vo = case
    V, F, r, pe, ge = m.build_patch_design_gpu(Lp, Wp, Lg, Wg, h, npx, npy, ngx, ngy, feed=feed, vertex_order=vo)
    Vo, Fo = eo.make_patch_with_ground_mesh(Lp, Wp, Lg, Wg, h, npx, npy, ngx, ngy, vertex_order=vo)
    ro = eo.build_rwg_interior(Vo, Fo)
    assert np.array_equal(V, Vo) and np.array_equal(F, Fo)
    assert r["Ne"] == ro["Ne"]
    for f in ("edge", "plusTri", "minusTri", "plusSign", "minusSign", "zSign"):
        assert np.array_equal(r[f], ro[f]), f
    for f in ("rp", "rm", "Ap", "Am", "len", "center"):
        assert np.array_equal(r[f], ro[f]), f
    assert pe == eo.pick_port_edge_by_point_and_layer(ro, (feed[0], feed[1], +h / 2), +1)
    assert ge == eo.pick_port_edge_by_point_and_layer(ro, (feed[0], feed[1], -h / 2), -1)
