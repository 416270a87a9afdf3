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


@pytest.mark.parametrize("lu_nb", [128, 256, 512])
def test_lu_symmetric_matches_general(lu_nb):
    """A bit-exactly symmetric Z (the symmetric gather's) is factored as
    L D L^T: the trailing updates form only the lower part and the outer
    panels' diagonal blocks, and the row panel comes from the lower part
    transposed; the diagonal blocks are factored as L D L^T with
    U^-1 = L^-T D^-1.  Its factors reproduce Z about as closely as the
    general factorization's (within 4x of its worst entry), in the upper and
    the lower triangle alike."""
    nat = importlib.import_module("matlab-cuda-efief-vs-cpu_b200._native")
    d = config1_design("grid")
    p = eo.build_problem(d)
    omega, k, _, _ = eo.physics(2.5e9, d.mu, d.eps)
    Z = oc.assemble_z(p["rwg"], p["prepack"], k, omega, d.mu, d.eps)
    Z = np.triu(Z) + np.triu(Z, 1).T
    assert np.array_equal(Z, Z.T)
    nat.lib().efie_debug_set_selftest_panel(lu_nb)
    try:
        sym = _lu(Z, True)
        nat.lib().efie_debug_disable_symmetric_lu(1)
        gen = _lu(Z, True)
    finally:
        nat.lib().efie_debug_disable_symmetric_lu(0)
        nat.lib().efie_debug_set_selftest_panel(0)
    n = Z.shape[0]
    zmax = np.abs(Z).max()

    def errs(LU):
        E = np.abs((np.tril(LU, -1) + np.eye(n)) @ np.triu(LU) - Z) / zmax
        return np.tril(E).max(), np.triu(E, 1).max()

    es, eg = errs(sym), errs(gen)
    assert max(eg) <= 5e-5
    assert max(es) <= 4 * max(eg), (es, eg)


@pytest.mark.parametrize("n,lu_nb", [(257, 128), (700, 256), (1300, 512), (1300, 128)])
def test_lu_symmetric_random(n, lu_nb):
    """Random complex symmetric, diagonally dominant matrices (partial last
    diagonal block and partial last outer panel): the L D L^T factors
    reproduce A to FP32 accuracy, with U = D L^T."""
    nat = importlib.import_module("matlab-cuda-efief-vs-cpu_b200._native")
    rng = np.random.default_rng(n + lu_nb)
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    A = A + A.T + np.diag(4.0 + 2.0j + rng.standard_normal(n))
    nat.lib().efie_debug_set_selftest_panel(lu_nb)
    try:
        LU = _lu(A, True)
    finally:
        nat.lib().efie_debug_set_selftest_panel(0)
    assert _residual(A, LU) <= 2e-6
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    DLt = np.diag(np.diag(U)) @ L.T
    assert np.abs(U - DLt).max() <= 1e-5 * np.abs(U).max()


@pytest.mark.parametrize("tiles", [(128, 128, 0), (128, 256, 0), (256, 128, 0), (256, 256, 1), (256, 256, 3)])
@pytest.mark.parametrize("n,lu_nb,sym", [(700, 256, False), (1300, 512, True), (1300, 128, True)])
def test_lu_tile_widths(tiles, n, lu_nb, sym):
    """The 256 x 128 tensor-core tile (a CTA pair per 128 complex columns)
    gives the same factors as the 256 x 256 tile to FP32 accuracy, for the
    panel chain's K = 64 updates and for the outer panels' updates, in the
    general and in the symmetric factorization; so do the resident, pipelined
    CTA pairs (third entry: 1 the chain updates, 3 also the outer panels'
    rectangular updates)."""
    nat = importlib.import_module("matlab-cuda-efief-vs-cpu_b200._native")
    rng = np.random.default_rng(n + lu_nb + tiles[0])
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    if sym:
        A = A + A.T
    A += np.diag(4.0 + 2.0j + rng.standard_normal(n))
    nat.lib().efie_debug_set_selftest_panel(lu_nb)
    try:
        ref = _lu(A, True)
        nat.lib().efie_debug_set_selftest_tiles(*tiles)
        got = _lu(A, True)
    finally:
        nat.lib().efie_debug_set_selftest_tiles(0, 0, 0)
        nat.lib().efie_debug_set_selftest_panel(0)
    assert _residual(A, got) <= 2e-6
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6
