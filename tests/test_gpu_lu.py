"""The hand-written complex128 LU / triangular solve against LAPACK on
random and structured matrices, including every blocking edge case."""

import numpy as np
import pytest
import scipy.linalg

from conftest import rel_err
from momwire_b200 import _lib

pytestmark = pytest.mark.gpu


def _factor_solve(A, B, device):
    import torch

    n = A.shape[0]
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).to(device)  # column-major
    Bd = torch.from_numpy(np.ascontiguousarray(B.T)).to(device)
    ws_bytes = _lib.load().mw_getrf_workspace_size(n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
    ipiv = torch.empty(max(n, 1), dtype=torch.int32, device=device)
    info = torch.zeros(2, dtype=torch.int32, device=device)
    _lib.call("mw_zgetrf", n, Ad.data_ptr(), n, ipiv.data_ptr(), info.data_ptr(), ws.data_ptr(), ws_bytes, None, None)
    _lib.call("mw_zgetrs", n, B.shape[1], Ad.data_ptr(), n, ipiv.data_ptr(), Bd.data_ptr(), n, None)
    return Ad.cpu().numpy().T, ipiv.cpu().numpy(), info.cpu().numpy(), Bd.cpu().numpy().T


@pytest.mark.parametrize("n", [1, 2, 3, 33, 63, 64, 65, 127, 128, 129, 300, 1000])
def test_lu_solve_random(n, cuda_device):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    B = rng.standard_normal((n, 5)) + 1j * rng.standard_normal((n, 5))
    LU, ipiv, info, X = _factor_solve(A, B, cuda_device)
    assert info[0] == 0 and info[1] == 0
    lu_ref, piv_ref = scipy.linalg.lu_factor(A)
    assert np.array_equal(ipiv, piv_ref + 1)  # same pivots as LAPACK
    assert rel_err(LU, lu_ref) < 1e-10
    assert rel_err(X, np.linalg.solve(A, B)) < 1e-9


@pytest.mark.parametrize("n,nrhs", [(300, 37), (650, 129)])
def test_lu_solve_many_right_hand_sides(n, nrhs, cuda_device):
    """Complex128 sweeps over several leaf CTAs with a partial last block and
    the fused next-block update."""
    rng = np.random.default_rng(n + nrhs)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    B = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    _LU, _ipiv, info, X = _factor_solve(A, B, cuda_device)
    assert info[0] == 0 and info[1] == 0
    assert rel_err(X, np.linalg.solve(A, B)) < 1e-9


def test_lu_pivoting_needed(cuda_device):
    """A matrix that fails without row interchanges."""
    A = np.array([[0, 1, 2], [1, 0, 3], [4, 5, 0]], dtype=np.complex128)
    B = np.eye(3, dtype=np.complex128)
    _LU, ipiv, info, X = _factor_solve(A, B, cuda_device)
    assert info[0] == 0
    assert rel_err(X, np.linalg.inv(A)) < 1e-14


def test_lu_exact_zero_pivot_reports_info(cuda_device):
    A = np.zeros((70, 70), dtype=np.complex128)
    A[np.arange(70), np.arange(70)] = 1.0
    A[65, 65] = 0.0
    _LU, _ipiv, info, _X = _factor_solve(A, np.ones((70, 1), dtype=np.complex128), cuda_device)
    assert info[0] == 66  # LAPACK convention: 1-based index of the zero pivot


def test_zgemm_transposes(cuda_device):
    import torch

    rng = np.random.default_rng(7)
    for ta, tb in [(0, 0), (1, 0), (0, 1), (1, 1)]:
        m, n, k = 37, 71, 130
        A = rng.standard_normal((k, m) if ta else (m, k)) + 1j * rng.standard_normal((k, m) if ta else (m, k))
        B = rng.standard_normal((n, k) if tb else (k, n)) + 1j * rng.standard_normal((n, k) if tb else (k, n))
        C0 = rng.standard_normal((m, n)) + 0j
        Ad = torch.from_numpy(np.ascontiguousarray(A.T)).to(cuda_device)
        Bd = torch.from_numpy(np.ascontiguousarray(B.T)).to(cuda_device)
        Cd = torch.from_numpy(np.ascontiguousarray(C0.T)).to(cuda_device)
        _lib.call("mw_zgemm", ta, tb, m, n, k, 2.0, 0.5, Ad.data_ptr(), A.shape[0], Bd.data_ptr(), B.shape[0],
                  -1.0, 0.0, Cd.data_ptr(), m, None)
        want = (2.0 + 0.5j) * ((A.T if ta else A) @ (B.T if tb else B)) - C0
        assert rel_err(Cd.cpu().numpy().T, want) < 1e-13
