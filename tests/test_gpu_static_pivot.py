"""Static pivoting of the mixed-precision factorisation.

mw_zgesv_mixed chooses pivots within each 128-row diagonal block (no
column-wide pivot search) and keeps that factorisation only when every
|L21| stays within its bound and the FP64 refinement reaches its tolerance;
otherwise it repeats the solve with partial pivoting.  These tests check
(1) solves through the C ABI on matrices that need no cross-block
interchange agree with partial pivoting and with numpy; (2) a matrix whose
diagonal blocks are nearly singular is rejected and solved by the fallback;
(3) the public solver's results on the golden cases and the 16 x 16 array
are unchanged, with the static factorisation kept."""

import ctypes as C

import numpy as np
import pytest

from cases import CASES
from conftest import golden, rel_err

import momwire_b200
from momwire_b200 import _lib

pytestmark = pytest.mark.gpu


def _zgesv_mixed(Z, B, device, mode):
    """X, iterations, pivoting used: one mw_zgesv_mixed through the C ABI."""
    import torch

    lib = _lib.load()
    n, nrhs = B.shape
    Zd = torch.from_numpy(np.ascontiguousarray(Z.T)).to(device)
    Z32 = torch.from_numpy(np.ascontiguousarray(Z.T.astype(np.complex64))).to(device)
    Bd = torch.from_numpy(np.ascontiguousarray(B.T)).to(device)
    Xd = torch.empty((nrhs, n), dtype=torch.complex128, device=device)
    ipiv = torch.empty(n, dtype=torch.int32, device=device)
    info = torch.zeros(4, dtype=torch.int32, device=device)
    wsb = lib.mw_zgesv_mixed_workspace_size(n, nrhs)
    ws = torch.empty(wsb, dtype=torch.uint8, device=device)
    it, corr = C.c_int32(0), C.c_double(0.0)
    prev = lib.mw_set_mixed_pivoting(mode)
    try:
        _lib.call("mw_zgesv_mixed", n, nrhs, Zd.data_ptr(), n, Z32.data_ptr(), n, ipiv.data_ptr(), Bd.data_ptr(), n,
                  Xd.data_ptr(), n, 1e-10, 10, ws.data_ptr(), wsb, info.data_ptr(), C.byref(it), C.byref(corr), None,
                  None)
    finally:
        lib.mw_set_mixed_pivoting(prev)
    return Xd.cpu().numpy().T, int(it.value), int(lib.mw_last_mixed_pivoting())


def _diag_heavy(n, rng):
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return A + np.eye(n) * (4.0 * np.sqrt(n))


@pytest.mark.parametrize("n,nrhs", [(1, 1), (127, 3), (128, 5), (129, 2), (300, 7), (1000, 64)])
def test_static_pivots_solve_like_partial_pivoting(n, nrhs, cuda_device):
    rng = np.random.default_rng(1000 + n)
    Z = _diag_heavy(n, rng)
    B = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    want = np.linalg.solve(Z, B)
    xs, _its, used_s = _zgesv_mixed(Z, B, cuda_device, 0)
    xp, _itp, used_p = _zgesv_mixed(Z, B, cuda_device, 1)
    assert used_s == 0 and used_p == 1
    assert rel_err(xs, want) < 1e-9
    assert rel_err(xp, want) < 1e-9


@pytest.mark.parametrize("n", [384, 300, 100, 38])
def test_static_pivots_within_the_block(n, cuda_device):
    """Interchanges that stay inside the diagonal blocks are made: each
    block's rows reversed, so that partial pivoting must swap within it
    (in the 32-column panels of a full block and of a partial last one)."""
    rng = np.random.default_rng(7)
    Z = _diag_heavy(n, rng)
    perm = np.concatenate([np.arange(min(b + 128, n) - 1, b - 1, -1) for b in range(0, n, 128)])
    Z = Z[perm]
    B = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
    x, _it, used = _zgesv_mixed(Z, B, cuda_device, 0)
    assert used == 0
    assert rel_err(x, np.linalg.solve(Z, B)) < 1e-9


def _swapped_blocks(n, rng):
    """100 I + 1e-3 noise with the two 128-row halves exchanged: every
    diagonal block holds only the noise, the large entries sit below it."""
    Z = 100.0 * np.eye(n) + 1e-3 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    return Z[np.concatenate([np.arange(128, 256), np.arange(0, 128)])]


def test_nearly_singular_blocks_fall_back(cuda_device):
    """|L21| grows far past the bound (~1e5): the static factorisation is
    rejected and the solve repeated with partial pivoting."""
    rng = np.random.default_rng(11)
    Z = _swapped_blocks(256, rng)
    B = rng.standard_normal((256, 4)) + 1j * rng.standard_normal((256, 4))
    x, _it, used = _zgesv_mixed(Z, B, cuda_device, 0)
    assert used == 2
    assert rel_err(x, np.linalg.solve(Z, B)) < 1e-9


def test_exact_zero_block_pivot_falls_back(cuda_device):
    """A diagonal block with an exactly zero column: the block is singular,
    so the static factorisation is rejected (the matrix itself is not)."""
    rng = np.random.default_rng(12)
    Z = _swapped_blocks(256, rng)
    Z[:128, 5] = 0.0
    B = rng.standard_normal((256, 2)) + 1j * rng.standard_normal((256, 2))
    x, _it, used = _zgesv_mixed(Z, B, cuda_device, 0)
    assert used == 2
    assert rel_err(x, np.linalg.solve(Z, B)) < 1e-9


def test_pivoting_mode_is_validated():
    lib = _lib.load()
    assert lib.mw_set_mixed_pivoting(5) == _lib.MW_ERR_INVALID
    prev = lib.mw_set_mixed_pivoting(1)
    assert lib.mw_set_mixed_pivoting(prev) == 1


def _zin(y):
    return 1.0 / np.diag(y)


@pytest.mark.parametrize("name", ["config1", "d2_junction_port", "d2_refl_normal", "d1_yagi", "d2_somm_radials",
                                  "array4x4"])
def test_solver_keeps_static_factorisation(name, cuda_device):
    g = golden(name)
    s = momwire_b200.BSplineSolver(**CASES[name](), precision="mixed")
    y = s.compute_port_solution().y
    assert _lib.load().mw_last_mixed_pivoting() in (0, 2)
    assert np.max(np.abs(_zin(y) - _zin(g["y"])) / np.abs(_zin(g["y"]))) <= 1e-6


def test_array16x16_static_pivots(cuda_device):
    from momwire_b200.workloads import dipole_array

    g = golden("array16x16")
    s = momwire_b200.BSplineSolver(**dipole_array(16, 16), precision="mixed")
    y = s.compute_port_solution().y
    assert _lib.load().mw_last_mixed_pivoting() == 0
    assert rel_err(y, g["y"]) < 1e-6
    assert np.max(np.abs(_zin(y) - _zin(g["y"])) / np.abs(_zin(g["y"]))) <= 1e-6
