"""GPU numerics of the complex64 LU (tcgen05 3xTF32 trailing update) against a
plain fp64/fp32 reference: the factors must reproduce A to FP32 accuracy and
agree with the CUDA-core (SIMT FP32) factorisation.  Tolerances:
||L U - A|| / ||A|| <= 2e-6 (1e-5 for the EFIE matrix) and ||LU_tc - LU_simt|| / ||LU_simt|| <= 1e-5."""
import ctypes as C
import importlib

import numpy as np
import pytest

import efie_oracle as eo
import oracle_c as oc
from conftest import config1_design

pytestmark = pytest.mark.gpu


def _lu(A, tc):
    nat = importlib.import_module("matlab-cuda-efief-vs-cpu_b200._native")
    A = np.asfortranarray(A.astype(np.complex128))
    LU = np.zeros_like(A, order="F")
    nat.check(nat.lib().efie_lu_selftest(nat.context(), A.shape[0], A.ctypes.data, 1 if tc else 0, LU.ctypes.data))
    return LU


def _residual(A, LU):
    L = np.tril(LU, -1) + np.eye(A.shape[0])
    U = np.triu(LU)
    return np.linalg.norm(L @ U - A) / np.linalg.norm(A)


@pytest.mark.parametrize("n", [257, 700, 1300])
def test_lu_random_diagonally_dominant(n):
    rng = np.random.default_rng(n)
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    A += np.diag(4.0 + 2.0j + rng.standard_normal(n))
    tc = _lu(A, True)
    simt = _lu(A, False)
    assert _residual(A, tc) <= 2e-6
    assert _residual(A, simt) <= 2e-6
    assert np.linalg.norm(tc - simt) / np.linalg.norm(simt) <= 1e-5


def test_lu_efie_matrix():
    d = config1_design("grid")
    p = eo.build_problem(d)
    omega, k, _, _ = eo.physics(2.5e9, d.mu, d.eps)
    Z = oc.assemble_z(p["rwg"], p["prepack"], k, omega, d.mu, d.eps)
    tc = _lu(Z, True)
    assert _residual(Z, tc) <= 1e-5
    torch = pytest.importorskip("torch")
    # plain PyTorch fp32 reference of the same op: L U in complex64 on the GPU
    L = torch.tril(torch.from_numpy(tc.astype(np.complex64)), -1) + torch.eye(Z.shape[0], dtype=torch.complex64)
    U = torch.triu(torch.from_numpy(tc.astype(np.complex64)))
    R = (L.cuda() @ U.cuda()).cpu().numpy()
    assert np.linalg.norm(R - Z) / np.linalg.norm(Z) <= 1e-5
