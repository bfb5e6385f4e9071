"""CPU oracle for the learned Sommerfeld surrogate's MLP.

TEST INFRASTRUCTURE ONLY.  Only ``tests/`` may import this module, as the
checker of the CUDA forward/backward kernels.  The product package
``momwire_b200`` never imports it.

The surrogate has no counterpart in the reference (which tabulates the
Sommerfeld remainder by quadrature); this is a plain float64 numpy statement
of the network the kernels implement: 5 -> 128 -> 128 -> 128 -> 128 -> 8,
exact-erf GELU, weights rounded to BF16 (round to nearest even), FP32
biases, mean-squared-error loss, and its analytic gradient.  Its own
gradient is checked against central finite differences in the tests.
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf

DIMS = [(5, 128), (128, 128), (128, 128), (128, 128), (128, 8)]  # (in, out)


def offsets():
    """[(w_off, b_off)] of the flat parameter vector [W_l (out x in), b_l]."""
    out, o = [], 0
    for i, n in DIMS:
        out.append((o, o + i * n))
        o += i * n + n
    return out, o


OFFSETS, N_PARAMS = offsets()


def bf16_round(x):
    """float32 -> nearest BF16 value (ties to even), returned as float32."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p, bf16=True):
    """[(W (out x in), b)] with W BF16-rounded when bf16."""
    p = np.asarray(p, dtype=np.float32)
    layers = []
    for (i, n), (wo, bo) in zip(DIMS, OFFSETS):
        W = p[wo:wo + i * n].reshape(n, i)
        layers.append(((bf16_round(W) if bf16 else W).astype(np.float64), p[bo:bo + n].astype(np.float64)))
    return layers


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward(X, p, keep=False):
    """Outputs (n x 8); with keep, also the per-layer (input, pre-activation)."""
    a = np.asarray(X, dtype=np.float64)
    cache = []
    layers = unpack(p)
    for li, (W, b) in enumerate(layers):
        z = a @ W.T + b
        cache.append((a, z))
        a = gelu(z) if li < len(layers) - 1 else z
    return (a, cache) if keep else a


def loss_and_grad(X, T, p):
    """Mean squared error over all outputs and its gradient with respect to
    every parameter (the BF16-rounded weights are the ones differentiated)."""
    out, cache = forward(X, p, keep=True)
    T = np.asarray(T, dtype=np.float64)
    n = out.size
    loss = float(np.sum((out - T) ** 2) / n)
    g = np.zeros(N_PARAMS)
    d = 2.0 * (out - T) / n
    layers = unpack(p)
    for li in range(len(layers) - 1, -1, -1):
        a_in, z = cache[li]
        if li < len(layers) - 1:
            d = d * gelu_grad(z)
        wo, bo = OFFSETS[li]
        i, nn = DIMS[li]
        g[wo:wo + i * nn] = (d.T @ a_in).ravel()
        g[bo:bo + nn] = d.sum(axis=0)
        d = d @ layers[li][0]
    return loss, g


def init_params(seed=0):
    """He-style initialisation (what the trainer starts from)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, dtype=np.float32)
    for (i, n), (wo, bo) in zip(DIMS, OFFSETS):
        p[wo:wo + i * n] = rng.standard_normal(i * n) * np.sqrt(2.0 / i)
    return p
