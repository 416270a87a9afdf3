"""Surrogate MLP and surrogate-guided adaptive sweeps.

CPU: the FP64 oracle of the network (finite-difference gradients, BF16
rounding, Adam) and the host-side sweep logic.  GPU: the CUDA forward,
backward and Adam kernels against the oracle (forward |dY| <= 1e-5 |Y|,
gradient |dg| <= 1e-4 |g|, Adam step <= 1e-6 relative), training on the GPU,
and the adaptive sweep against the dense plain sweep.
"""
import importlib

import numpy as np
import pytest

import mlp_oracle as mo

PKG = "matlab-cuda-efief-vs-cpu_b200"


def _sur():
    return importlib.import_module(PKG + ".surrogate")


SMALL = dict(n_in=5, n_hidden=32, n_layers=2, n_out=2)


def _shapes(c):
    return mo.layer_shapes(c["n_in"], c["n_hidden"], c["n_layers"], c["n_out"])


def _rand_params(shapes, seed):
    rng = np.random.default_rng(seed)
    out = []
    for fi, fo in shapes:
        a = 1.0 / np.sqrt(fi)
        out.append(rng.uniform(-a, a, fi * fo))
        out.append(rng.uniform(-a, a, fo))
    return np.concatenate(out).astype(np.float32)


# ---------------------------------------------------------------------------
# CPU: the oracle itself
# ---------------------------------------------------------------------------
def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e-3], dtype=np.float32)
    r = mo.bf16_round(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: ties go to the even mantissa (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2 ** -6) and r[3] == 1.0
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-3) <= 2 ** -8 * 3.0e-3


def test_oracle_gradient_matches_finite_differences():
    shapes = _shapes(SMALL)
    p = _rand_params(shapes, 3)
    rng = np.random.default_rng(4)
    X = rng.standard_normal((16, 5)).astype(np.float32)
    T = rng.standard_normal((16, 2)).astype(np.float32)
    # with weights that are exact BF16 values the loss is smooth in the biases;
    # check the bias gradients by central differences in FP64
    layers = mo.unpack(p.copy(), shapes)
    _, g = mo.loss_grad(p, shapes, X, T)
    o = 0
    for (W, b), (fi, fo) in zip(layers, shapes):
        o += fi * fo
        for j in range(min(fo, 4)):
            h = 1e-3
            pp, pm = p.astype(np.float64).copy(), p.astype(np.float64).copy()
            pp[o + j] += h
            pm[o + j] -= h
            lp = np.mean((mo.forward(pp, shapes, X) - T) ** 2)
            lm = np.mean((mo.forward(pm, shapes, X) - T) ** 2)
            assert abs((lp - lm) / (2 * h) - g[o + j]) <= 1e-4 * max(1.0, abs(g[o + j]))
        o += fo


def test_oracle_adam_first_step_is_signed_lr():
    w = np.zeros(4)
    g = np.array([1.0, -2.0, 0.5, -1e-3])
    w1, m, v = mo.adam_step(w, g, np.zeros(4), np.zeros(4), 1, lr=0.01)
    assert np.allclose(w1, -0.01 * np.sign(g), rtol=1e-4)


def test_refine_min_and_interpolant():
    s = _sur()
    f = np.linspace(0.0, 1.0, 11)
    y = (f - 0.437) ** 2
    assert abs(s._refine_min(f, y) - 0.437) < 1e-12
    fs = np.linspace(0.0, 1.0, 9)
    z = np.sin(fs) + 1j * fs ** 2
    fq = np.linspace(0.0, 1.0, 101)
    zi = s._interp_correction(fs, z, fq)
    assert np.abs(zi - (np.sin(fq) + 1j * fq ** 2)).max() < 2e-3
    assert np.allclose(s._interp_correction(fs, z, fs), z)


def test_target_round_trip():
    s = _sur()
    z = np.array([1e-3 + 2e-4j, 0.27j, 35.2 + 19.4j, -3.0 - 1e-9j, 400.0])
    assert np.allclose(s.target_to_zin(s.zin_to_target(z)), z, rtol=1e-6, atol=0)


def test_design_sampling_and_features():
    s = _sur()
    ds = s.sample_designs(50, seed=1)
    for d in ds:
        assert 25e-3 <= d.W <= 45e-3 and 20e-3 <= d.L <= 40e-3 and 0.8e-3 <= d.h <= 3.2e-3
        assert abs(d.feed) <= d.L / 3
        X = s.features(d, d.band(5))
        assert np.all(np.abs(X) <= 1.0 + 1e-6)
        assert np.allclose(X[[0, -1], 4], [-1.0, 1.0])


# ---------------------------------------------------------------------------
# GPU: kernels against the oracle
# ---------------------------------------------------------------------------
@pytest.fixture
def small_net():
    s = _sur()
    net = s.Surrogate(**SMALL, seed=7)
    yield net
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 37, 300])
def test_forward_matches_oracle(small_net, n):
    shapes = _shapes(SMALL)
    p = _rand_params(shapes, n)
    small_net.set_params(p)
    X = np.random.default_rng(n).standard_normal((n, 5)).astype(np.float32)
    Y = small_net.forward(X)
    Yo = mo.forward(p, shapes, X)
    assert np.abs(Y - Yo).max() <= 1e-5 * max(1.0, np.abs(Yo).max())


@pytest.mark.gpu
def test_gradients_match_oracle_full_size():
    s = _sur()
    net = s.Surrogate(seed=11)   # 5 -> 4 x 256 (SiLU) -> 3
    shapes = mo.layer_shapes(5, 256, 4, 3)
    p = net.get_params()
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (700, 5)).astype(np.float32)
    T = rng.standard_normal((700, 3)).astype(np.float32)
    loss, g = net.loss_grad(X, T)
    lo, go = mo.loss_grad(p, shapes, X, T)
    assert abs(loss - lo) <= 1e-5 * lo
    # per layer: relative to the layer's gradient norm
    o = 0
    for fi, fo in shapes:
        for size in (fi * fo, fo):
            a, b = g[o:o + size], go[o:o + size]
            assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b) + 1e-12
            o += size
    net.close()


@pytest.mark.gpu
def test_adam_step_matches_oracle(small_net):
    shapes = _shapes(SMALL)
    p = _rand_params(shapes, 21)
    small_net.set_params(p)
    rng = np.random.default_rng(6)
    X = rng.uniform(-1, 1, (64, 5)).astype(np.float32)
    T = rng.standard_normal((64, 2)).astype(np.float32)
    _, g = small_net.loss_grad(X, T)
    small_net.train(X, T, epochs=1, batch=64, lr=1e-2)
    p1 = small_net.get_params()
    w1, _, _ = mo.adam_step(p.astype(np.float64), g.astype(np.float64), 0.0, 0.0, 1, lr=1e-2)
    # the step's gradient sums the same rows in another order: compare where
    # |g| is well above Adam's eps
    big = np.abs(g) > 1e-5
    assert np.abs(p1 - w1)[big].max() <= 1e-6
    assert np.abs(p1 - p).max() <= 1.0001e-2


@pytest.mark.gpu
def test_training_reduces_loss():
    s = _sur()
    net = s.Surrogate(n_hidden=64, n_layers=3, n_out=2, seed=3)
    rng = np.random.default_rng(8)
    X = rng.uniform(-1, 1, (4096, 5)).astype(np.float32)
    T = np.stack([np.sin(2 * X[:, 4] + X[:, 0]) * X[:, 1], np.cos(3 * X[:, 4]) + 0.3 * X[:, 2]], 1).astype(np.float32)
    hist = net.train(X, T, epochs=60, batch=512, lr=3e-3)
    assert np.all(np.isfinite(hist))
    assert hist[-1] < 0.05 * hist[0]
    # the loss the network reports after training agrees with its forward pass
    loss, _ = net.loss_grad(X, T)
    assert abs(loss - np.mean((net.forward(X) - T) ** 2)) <= 1e-5 * loss + 1e-9
    net.close()


@pytest.mark.gpu
def test_adaptive_sweep_beats_uniform_budget():
    """A surrogate trained on the GPU from solver samples of a design family
    finds the |S11| minimum of held-out designs with far fewer EFIE solves than
    the dense 201-point sweep, and more precisely than the method without the
    network at the same number of solves (uniform points + cubic interpolation).
    Coarse meshes (patch 3 mm, ground 6 mm; Ne ~ 330-920) keep the test short."""
    s = _sur()
    train = s.sample_designs(100, seed=1, pitch=3e-3, ground_pitch=6e-3)
    X, T = s.generate_samples(train, 40, seed=2)
    net = s.Surrogate(seed=3)
    hist = net.train(X, T, epochs=400, batch=512, lr=2e-3)
    net.train(X, T, epochs=200, batch=512, lr=3e-4)
    assert hist[-1] < 0.2 * hist[0]
    test = s.sample_designs(8, seed=99, pitch=3e-3, ground_pitch=6e-3)
    solves, err_ad, err_un = [], [], []
    for d in test:
        plan = s.design_plan(d)
        dn = s.dense_sweep(d, 201, plan)
        step = d.band(201)[1] - d.band(201)[0]
        ad = s.adaptive_sweep(d, net, plan)
        un = s.uniform_sweep_estimate(d, ad["solves"], plan)
        plan.close()
        solves.append(ad["solves"])
        err_ad.append(abs(ad["f_min"] - dn["f_min"]) / step)
        err_un.append(abs(un["f_min"] - dn["f_min"]) / step)
    net.close()
    err_ad, err_un = np.array(err_ad), np.array(err_un)
    # most designs resolve without the dense fallback, at a fraction of its solves
    assert np.median(solves) <= 48
    # the solved points locate the minimum to a fraction of the dense grid step,
    # at least as well as the same number of uniform solves on nearly every design
    assert np.median(err_ad) <= 0.5
    assert np.sum(err_ad <= err_un + 0.5) >= 6


@pytest.mark.gpu
def test_gradients_are_bit_reproducible():
    """The weight gradients' K-split partial products are added in a fixed
    order (no atomics), as are the bias gradients' column sums: the same
    minibatch gives the same gradient bit for bit."""
    s = _sur()
    net = s.Surrogate(seed=4)
    rng = np.random.default_rng(9)
    X = rng.uniform(-1, 1, (1500, 5)).astype(np.float32)    # three K chunks of 512 rows
    T = rng.standard_normal((1500, 3)).astype(np.float32)
    l1, g1 = net.loss_grad(X, T)
    l2, g2 = net.loss_grad(X, T)
    assert l1 == l2 and np.array_equal(g1, g2)
    net.close()
