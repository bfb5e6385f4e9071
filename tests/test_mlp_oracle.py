"""The surrogate MLP's CPU oracle (its analytic gradient against finite
differences) and the host-side feature map and domain of the surrogate."""

import math

import numpy as np

from oracle import mlp_oracle as M

from momwire_b200 import _lib, surrogate


def test_param_layout_matches_library():
    assert M.N_PARAMS == 51336
    assert int(_lib.load().mw_mlp_param_count()) == M.N_PARAMS
    assert surrogate.he_init(0).size == M.N_PARAMS


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-20, 65504.0], dtype=np.float32)
    r = M.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0  # ties to even
    assert r[2] == np.float32(1.0 + 2 ** -7)
    assert abs(r[3] - (-3.140625)) < 1e-7
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = M.init_params(2) * 0.5
    X = rng.uniform(-1, 1, (7, 5))
    T = rng.standard_normal((7, 8))
    _loss, g = M.loss_and_grad(X, T, p)
    # perturb biases (not BF16-rounded) and a few weights along a smooth
    # direction in float64 by differentiating the oracle's own float64 path
    idx = [M.OFFSETS[0][1] + 3, M.OFFSETS[2][1] + 7, M.OFFSETS[4][1] + 5]
    for i in idx:
        h = 1e-3
        pp, pm = p.astype(np.float64).copy(), p.astype(np.float64).copy()
        pp[i] += h
        pm[i] -= h
        lp = np.sum((M.forward(X, pp.astype(np.float32)) - T) ** 2) / T.size
        lm = np.sum((M.forward(X, pm.astype(np.float32)) - T) ** 2) / T.size
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-4 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_weight_gradient_matches_finite_differences_unrounded():
    """Weights enter BF16-rounded, so differentiate the unrounded network."""
    rng = np.random.default_rng(3)
    p = M.init_params(4) * 0.5
    X = rng.uniform(-1, 1, (5, 5))
    T = rng.standard_normal((5, 8))

    def loss(pv):
        a = X
        layers = M.unpack(pv, bf16=False)
        for li, (W, b) in enumerate(layers):
            z = a @ W.T + b
            a = M.gelu(z) if li < len(layers) - 1 else z
        return np.sum((a - T) ** 2) / T.size

    # analytic gradient of the unrounded network = oracle gradient with
    # weights that are already exactly BF16
    pr = p.copy()
    for (i, n), (wo, _bo) in zip(M.DIMS, M.OFFSETS):
        pr[wo:wo + i * n] = M.bf16_round(pr[wo:wo + i * n])
    _l, g = M.loss_and_grad(X, T, pr)
    pr64 = pr.astype(np.float64)
    for i in [M.OFFSETS[1][0] + 11, M.OFFSETS[3][0] + 2000, M.OFFSETS[4][0] + 17]:
        h = 1e-6
        pp, pm = pr64.copy(), pr64.copy()
        pp[i] += h
        pm[i] -= h
        fd = (loss(pp) - loss(pm)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_features_and_domain():
    rho = np.array([0.0, 1.0, 3.9])
    h = np.array([0.02, 1.0, 0.1])
    eps = np.array([10 - 1j, 40 - 500j, 3 - 0.01j])
    f = np.array([3e6, 14e6, 30e6])
    x = surrogate.features(rho, h, eps, f)
    assert x.shape == (3, 5) and x.dtype == np.float32
    assert np.all(np.abs(x) <= 1.0 + 1e-6)
    assert abs(x[0, 1] - 1.0) < 1e-6  # theta = 90 deg
    assert np.all(surrogate.in_domain(rho, h, eps, f))
    assert not surrogate.in_domain(5.0, 0.1, 10 - 1j, 1e7)
    assert not surrogate.in_domain(1.0, 0.001, 10 - 1j, 1e7)
    assert not surrogate.in_domain(1.0, 0.1, 10 - 1j, 1e8)


def test_training_distribution_stays_in_domain():
    rng = np.random.default_rng(0)
    rho, h, eps, f = surrogate.sample_domain(20000, rng)
    assert np.all(surrogate.in_domain(rho, h, eps, f))
    assert np.all(np.abs(surrogate.features(rho, h, eps, f)) <= 1.0 + 1e-5)
    assert math.isclose(float(np.median(np.log10(np.abs(eps)))), 1.5, abs_tol=1.0)
