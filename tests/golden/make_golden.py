"""Generates the golden vectors in tests/golden by running the reference's own
CUDA MEX code (compiled unmodified against the fake mex shim, oracle/_ref)
on a GPU.  Run once on a CUDA machine:

    make -C oracle && python tests/golden/make_golden.py [outdir]

Inputs are built with the oracle's restatement of the reference's MATLAB
producers (mesh, RWG, ports, precompute/pack), so the fixtures pin both the
oracle's assembly and its solve against the reference's GPU code.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import efie_oracle as eo  # noqa: E402
import ref_mex  # noqa: E402
from conftest import small_design  # noqa: E402


def main(out):
    os.makedirs(out, exist_ok=True)
    cases = {
        "small_grid_gpu": small_design("grid"),
        "small_ref_gpu": small_design("reference"),
        "small_grid_accurate": small_design("grid", opts=eo.DEFAULT_OPTS_ACCURATE, npx=3, npy=2, ngx=4, ngy=4),
    }
    for name, d in cases.items():
        p = eo.build_problem(d)
        omega, k, _, _ = eo.physics(2.4e9, d.mu, d.eps)
        Z, V = ref_mex.ggassemble(p, k, omega, d.mu, d.eps)
        np.savez_compressed(os.path.join(out, "ggassemble_%s.npz" % name), Z=Z, Vrhs=V, k=k, omega=omega)
        print(name, Z.shape)
        if name == "small_grid_gpu":
            Zc, Vc = ref_mex.gassemble(p, k, omega, d.mu, d.eps, 0.2)
            np.savez_compressed(os.path.join(out, "gassemble_small_grid.npz"), Z=Zc, Vrhs=Vc, k=k, omega=omega)
            Zin, S11 = ref_mex.patch_sweep_cuda(p, d.freqs)
            np.savez_compressed(os.path.join(out, "patch_sweep_cuda_small_grid.npz"), Zin=Zin, S11=S11,
                                freqs=d.freqs)
    d = eo.reference_sweep_design()
    p = eo.build_problem(d)
    Zin, S11 = ref_mex.patch_sweep_fastquad(p, d.freqs)
    np.savez_compressed(os.path.join(out, "patch_sweep_fastquad_refdesign.npz"), Zin=Zin, S11=S11,
                        freqs=d.freqs, freq_idx=np.array([0, 20, 40]))
    print("refdesign Zin[0]", Zin[0])


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
