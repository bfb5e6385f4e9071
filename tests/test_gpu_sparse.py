"""Sparse gathers of the port and KCL algebra (mw_csr_mm_c128) against
scipy.sparse, and the host CSR builder."""

import numpy as np
import pytest
import scipy.sparse

from conftest import rel_err

from momwire_b200 import _lib
from momwire_b200.bspline import _csr


def _coo(rng, n_rows, n_cols, nnz):
    r = rng.integers(0, n_rows, nnz)
    c = rng.integers(0, n_cols, nnz)
    v = rng.standard_normal(nnz) + 1j * rng.standard_normal(nnz)
    return r, c, v


def test_csr_builder_matches_scipy():
    rng = np.random.default_rng(7)
    r, c, v = _coo(rng, 9, 30, 40)
    ptr, col, val = _csr(r, c, v, 9)
    S = scipy.sparse.csr_matrix((val, col, ptr), shape=(9, 30)).toarray()
    want = scipy.sparse.coo_matrix((v, (r, c)), shape=(9, 30)).toarray()
    np.testing.assert_allclose(S, want, rtol=0, atol=1e-15)
    ptr, col, val = _csr(np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.int64), np.zeros(0), 4)
    assert list(ptr) == [0, 0, 0, 0, 0] and col.size == 0


@pytest.mark.gpu
@pytest.mark.parametrize("n_out,n,ncols,nnz", [(1, 5, 1, 3), (37, 400, 17, 120), (256, 10496, 256, 768),
                                               (50, 300, 3, 0)])
def test_csr_mm_matches_scipy(n_out, n, ncols, nnz, cuda_device):
    import torch

    rng = np.random.default_rng(n_out + nnz)
    r, c, v = _coo(rng, n_out, n, nnz)
    ptr, col, val = _csr(r, c, v, n_out)
    X = rng.standard_normal((n, ncols)) + 1j * rng.standard_normal((n, ncols))
    dev = cuda_device
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (ptr, col, val.view(np.float64))]
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(dev)  # column-major n x ncols
    Yd = torch.full((ncols, n_out), 7.0 + 0j, dtype=torch.complex128, device=dev)
    _lib.call("mw_csr_mm_c128", n_out, ncols, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), Xd.data_ptr(), n,
              Yd.data_ptr(), n_out, None)
    Y = Yd.cpu().numpy().T
    want = scipy.sparse.coo_matrix((v, (r, c)), shape=(n_out, n)) @ X
    if nnz:
        assert rel_err(Y, want) < 1e-14
    else:
        assert not Y.any()
