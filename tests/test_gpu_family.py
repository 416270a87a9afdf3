"""Design families swept with several designs in flight (surrogate.sweep_family):
each worker thread owns a library context and stream, meshes its designs on
the GPU and sweeps them.  Every design's Zin must equal the same design swept
alone on the process context (bit for bit: the sweeps share nothing), and
the GPU-meshed design must equal the host-meshed one."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PKG = "matlab-cuda-efief-vs-cpu_b200"


def test_concurrent_family_sweep_matches_designs_swept_alone():
    sur = importlib.import_module(PKG + ".surrogate")
    designs = sur.sample_designs(5, seed=7)          # coarse pitch: Ne of a few hundred
    nf = 9
    out = sur.sweep_family(designs, nf, workers=3)
    for d, (Ne, Zin) in zip(designs, out):
        xh = sur.design_inputs(d, device=False)
        xd = sur.design_inputs(d, device=True)
        assert xh["Ne"] == xd["Ne"] == Ne
        for f in ("edge", "plusTri", "minusTri", "plusSign", "minusSign", "rp", "rm", "Ap", "Am", "len"):
            assert np.array_equal(xh["rwg"][f], xd["rwg"][f]), f
        assert (xh["pe"], xh["ge"]) == (xd["pe"], xd["ge"])
        plan = sur.design_plan(d, inputs=xh, nfreq=nf)   # the same batches as in the family
        Z1, _ = plan.run(d.band(nf))
        plan.close()
        assert np.array_equal(Zin, Z1)
