"""CPU tests: the native boundary-data producers (mesh, RWG topology, port
pick, precompute/pack) against the oracle's restatement of the reference's
MATLAB code -- integers bit-exact, floats bit-exact as well."""
import numpy as np
import pytest

import efie_oracle as eo
from conftest import pkg

CASES = [
    (30e-3, 38e-3, 60e-3, 60e-3, 1.6e-3, 12, 10, 16, 16),       # 38x30 mm patch, 12x10 / 16x16
    (20.1e-3, 20.1e-3, 0.2, 0.2, 1.59e-3, 8, 6, 12, 12),         # the reference's own sweep mesh
    (10e-3, 7e-3, 20e-3, 25e-3, 1e-3, 1, 1, 1, 2),               # smallest ragged case
]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("order", ["reference", "grid"])
def test_mesh_and_rwg_bit_exact(case, order):
    m = pkg()
    V, F, pidx, gidx = m.make_patch_with_ground_mesh(*case, vertex_order=order)
    Vo, Fo = eo.make_patch_with_ground_mesh(*case, vertex_order=order)
    assert np.array_equal(V, Vo) and np.array_equal(F, Fo)
    assert pidx[0] == 1 and gidx[-1] == F.shape[0]
    rwg = m.build_rwg_interior({"V": V, "F": F})
    ro = eo.build_rwg_interior(Vo, Fo)
    assert rwg["Ne"] == ro["Ne"]
    for k in ("edge", "plusTri", "minusTri", "plusSign", "minusSign", "zSign"):
        assert rwg[k].dtype == np.int32
        assert np.array_equal(rwg[k], ro[k]), k
    for k in ("rp", "rm", "Ap", "Am", "len", "center"):
        assert np.array_equal(rwg[k], ro[k]), k
    for layer, z in ((1, case[4] / 2), (-1, -case[4] / 2)):
        p = (0.0, -0.2 * case[0], z)
        assert m.pick_port_edge_by_point_and_layer(rwg, p, layer) == eo.pick_port_edge_by_point_and_layer(ro, p, layer)


@pytest.mark.parametrize("opts", [eo.DEFAULT_OPTS_GPU, eo.DEFAULT_OPTS_ACCURATE,
                                  dict(quad_order=eo.DUNAVANT7, near_sing_eps=1.5, self_subdiv=1, near_subdiv=0,
                                       near_order=1)])
def test_precompute_pack_bit_exact(opts):
    m = pkg()
    V, F = eo.make_patch_with_ground_mesh(16e-3, 12e-3, 30e-3, 30e-3, 1.6e-3, 4, 3, 6, 6, "grid")
    pre = m.efie_precompute_pack({"V": V, "F": F}, opts)
    po = eo.efie_precompute_pack(V, F, opts)
    for k, v in po.items():
        a = np.asarray(pre[k])
        assert a.shape == np.shape(v), k
        assert np.array_equal(a, np.asarray(v)), k


def test_quad_rule_sizes():
    m = pkg()
    assert [m.quad_rule_size(o) for o in (1, 2, 3, 4, 6, eo.DUNAVANT7)] == [1, 3, 6, 6, 6, 7]


def test_port_on_empty_layer_raises():
    m = pkg()
    V, F, _, _ = m.make_patch_with_ground_mesh(*CASES[2], vertex_order="grid")
    rwg = m.build_rwg_interior({"V": V, "F": F})
    with pytest.raises(m.MexError) as e:
        m.pick_port_edge_by_point_and_layer(rwg, (0, 0, 0), 5)
    assert e.value.identifier == "mex:port"
