"""Surrogate MLP kernels on the GPU: hand-written forward/backward/Adam
against the float64 numpy oracle, tensor-core inference against the FP32
forward, and the quadrature data path."""

import numpy as np
import pytest

from oracle import mlp_oracle as M

from momwire_b200 import _lib, surrogate

pytestmark = pytest.mark.gpu


def _dev(a, device, dtype=None):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.to(device=device, dtype=dtype) if dtype is not None else t.to(device)


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


def test_forward_and_gradient_match_oracle(cuda_device):
    import torch

    rng = np.random.default_rng(7)
    p = (M.init_params(5) * 0.5).astype(np.float32)
    p[M.OFFSETS[0][1]:M.OFFSETS[0][1] + 128] = rng.standard_normal(128).astype(np.float32) * 0.1
    n = 300
    X = rng.uniform(-1, 1, (n, 5)).astype(np.float32)
    T = rng.standard_normal((n, 8)).astype(np.float32)
    model = surrogate.Surrogate(p, cuda_device)
    y = model.predict_fp32(X).cpu().numpy()
    want = M.forward(X, p)
    assert np.max(np.abs(y - want)) <= 1e-5 * np.max(np.abs(want))
    lib = _lib.load()
    wsb = lib.mw_mlp_train_workspace_size(n)
    ws = torch.empty(wsb, dtype=torch.uint8, device=cuda_device)
    g = torch.empty(M.N_PARAMS, dtype=torch.float32, device=cuda_device)
    loss = torch.zeros(1, dtype=torch.float32, device=cuda_device)
    Xd, Td = _dev(X, cuda_device), _dev(T, cuda_device)
    _lib.call("mw_mlp_grad", n, Xd.data_ptr(), Td.data_ptr(), model.pbf.data_ptr(), model.p32.data_ptr(),
              g.data_ptr(), loss.data_ptr(), ws.data_ptr(), wsb, _stream())
    l_want, g_want = M.loss_and_grad(X, T, p)
    assert abs(float(loss.item()) - l_want) <= 1e-5 * l_want
    gg = g.cpu().numpy()
    for (i, nn), (wo, bo) in zip(M.DIMS, M.OFFSETS):
        for a, b in ((wo, bo), (bo, bo + nn)):
            assert np.max(np.abs(gg[a:b] - g_want[a:b])) <= 1e-4 * np.max(np.abs(g_want[a:b])) + 1e-9


def test_tensor_core_inference_matches_fp32_forward(cuda_device):
    rng = np.random.default_rng(11)
    p = (M.init_params(9) * 0.6).astype(np.float32)
    model = surrogate.Surrogate(p, cuda_device)
    for n in (1, 127, 128, 1000, 40000):
        X = rng.uniform(-1, 1, (n, 5)).astype(np.float32)
        y_tc = model.predict(X).cpu().numpy()
        y32 = model.predict_fp32(X).cpu().numpy()
        assert int(model.err.item()) == 0
        assert np.max(np.abs(y_tc - y32)) <= 2e-4 * np.max(np.abs(y32)), n


def test_adam_training_reduces_loss(cuda_device):
    """A few hundred Adam steps on a smooth 8-output target of the features."""
    import torch

    rng = np.random.default_rng(2)
    n = 16384
    X = rng.uniform(-1, 1, (n, 5)).astype(np.float32)
    T = np.stack([np.sin(1.5 * X[:, i % 5] + 0.3 * X[:, (i + 1) % 5]) for i in range(8)], axis=1).astype(np.float32)
    Xd, Td = _dev(X, cuda_device), _dev(T, cuda_device)
    model = surrogate.Surrogate(surrogate.he_init(0), cuda_device)
    lib = _lib.load()
    B = 1024
    wsb = lib.mw_mlp_train_workspace_size(B)
    ws = torch.empty(wsb, dtype=torch.uint8, device=cuda_device)
    m = torch.zeros(M.N_PARAMS, device=cuda_device)
    v = torch.zeros(M.N_PARAMS, device=cuda_device)
    loss = torch.zeros(1, device=cuda_device)
    first = None
    for step in range(1, 401):
        rows = torch.randint(0, n, (B,), device=cuda_device, dtype=torch.int64)
        loss.zero_()
        _lib.call("mw_mlp_train_step", B, Xd.data_ptr(), Td.data_ptr(), rows.data_ptr(), model.p32.data_ptr(),
                  model.pbf.data_ptr(), m.data_ptr(), v.data_ptr(), step, 1e-3, 0.9, 0.999, 1e-8, loss.data_ptr(),
                  ws.data_ptr(), wsb, _stream())
        if first is None:
            first = float(loss.item())
    last = float(loss.item())
    assert last < 0.05 * first, (first, last)


def test_per_node_eps_quadrature_matches_uniform(cuda_device):
    from momwire_b200 import sommerfeld as P

    rng = np.random.default_rng(4)
    rho = rng.uniform(0, 2, 64)
    h = rng.uniform(0.02, 2, 64)
    eps = 13 - 6.4j
    a = surrogate.quadrature_surfaces(rho, h, np.full(64, eps), cuda_device).cpu().numpy()
    import torch

    r1 = np.hypot(rho, h)
    th = np.arctan2(h, rho)
    d = _dev(np.stack([r1, rho, h, th]), cuda_device)
    out = torch.empty((64, 4), dtype=torch.complex128, device=cuda_device)
    ws = torch.empty(256, dtype=torch.uint8, device=cuda_device)
    _lib.call("mw_somm_surfaces", 64, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), eps.real,
              eps.imag, P.K2_REF, surrogate.OMEGA_REF, surrogate.MU0_GRID, 1e-6, out.data_ptr(), ws.data_ptr(),
              _stream())
    assert np.array_equal(a, out.cpu().numpy())
