"""The tensor-core complex update (tcgen05, 3xTF32) against a complex128
product on the host: ragged tile edges, several K stages, one and many
tiles per SM."""

import numpy as np
import pytest

from momwire_b200 import _lib

pytestmark = pytest.mark.gpu


def _run(m, n, k, seed, device):
    import torch

    rng = np.random.default_rng(seed)
    A = (rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))).astype(np.complex64)
    B = (rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))).astype(np.complex64)
    C = (rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))).astype(np.complex64)
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).to(device)  # column-major
    Bd = torch.from_numpy(np.ascontiguousarray(B.T)).to(device)
    Cd = torch.from_numpy(np.ascontiguousarray(C.T)).to(device)
    wsb = _lib.load().mw_cgemm_tc_workspace_size(m, n, k)
    ws = torch.empty(wsb, dtype=torch.uint8, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    _lib.call("mw_cgemm_tc_sub", m, n, k, Ad.data_ptr(), m, Bd.data_ptr(), k, Cd.data_ptr(), m, ws.data_ptr(), wsb,
              status.data_ptr(), None)
    got = Cd.cpu().numpy().T
    assert int(status.item()) == 0
    want = C.astype(np.complex128) - A.astype(np.complex128) @ B.astype(np.complex128)
    scale = np.abs(A).max() * np.abs(B).max() * k + np.abs(C).max()
    return float(np.abs(got - want).max() / scale)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (64, 256, 16), (70, 300, 64), (300, 513, 33), (1000, 1000, 64),
                                   (2500, 700, 128)])
def test_tc_update_matches_complex128(m, n, k, cuda_device):
    err = _run(m, n, k, m + n + k, cuda_device)
    # 3xTF32 keeps fp32-level accuracy: well below TF32's 2^-11
    assert err < 2e-6, err
