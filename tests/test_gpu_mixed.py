"""Mixed-precision path: complex64 tensor-core LU and FP64 refinement.

The bar is the one the fp64 drop-in is measured against: every port
impedance within |dZin|/|Zin| <= 1e-6 of the reference (complex128 LAPACK),
and Y within 1e-6 relative."""

import numpy as np
import pytest
import scipy.linalg

from cases import BIG_CASES, CASES
from conftest import golden, rel_err

import momwire_b200
from momwire_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 5, 64, 65, 200, 777])
def test_cgetrf_cgetrs_random(n, cuda_device):
    import torch

    rng = np.random.default_rng(100 + n)
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    A += np.eye(n, dtype=np.complex64) * 2  # keep it comfortably conditioned
    B = (rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))).astype(np.complex64)
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).to(cuda_device)
    Bd = torch.from_numpy(np.ascontiguousarray(B.T)).to(cuda_device)
    lib = _lib.load()
    wsb = lib.mw_cgetrf_workspace_size(n, 3)
    ws = torch.empty(wsb, dtype=torch.uint8, device=cuda_device)
    ipiv = torch.empty(n, dtype=torch.int32, device=cuda_device)
    info = torch.zeros(2, dtype=torch.int32, device=cuda_device)
    _lib.call("mw_cgetrf", n, Ad.data_ptr(), n, ipiv.data_ptr(), info.data_ptr(), ws.data_ptr(), wsb, 3, None, None)
    _lib.call("mw_cgetrs", n, 3, Ad.data_ptr(), n, ipiv.data_ptr(), Bd.data_ptr(), n, ws.data_ptr(), wsb, None)
    inf = info.cpu().numpy()
    assert inf[0] == 0 and inf[1] == 0
    X = Bd.cpu().numpy().T.astype(np.complex128)
    want = scipy.linalg.solve(A.astype(np.complex128), B.astype(np.complex128))
    cond = np.linalg.cond(A.astype(np.complex128))
    assert rel_err(X, want) < 50 * cond * 6e-8


def _zin(y):
    return 1.0 / np.diag(y)


@pytest.mark.parametrize("name", ["config1", "d2_junction", "d2_junction_port", "d2_refl_normal", "d2_ek",
                                  "d2_mixed_radius_kink"])
def test_mixed_matches_reference(name, cuda_device):
    g = golden(name)
    s = momwire_b200.BSplineSolver(**CASES[name](), precision="mixed")
    sol = s.compute_port_solution()
    assert rel_err(sol.y, g["y"]) < 1e-6
    assert np.max(np.abs(_zin(sol.y) - _zin(g["y"])) / np.abs(_zin(g["y"]))) <= 1e-6
    assert s.last_refinement["last_correction"] <= 1e-7


def test_mixed_array16x16(cuda_device):
    """The 16x16 dipole array (10,496 unknowns, 256 ports) through the
    tensor-core factorisation with FP64 refinement."""
    g = golden("array16x16")
    s = momwire_b200.BSplineSolver(**BIG_CASES["array16x16"](), precision="mixed")
    sol = s.compute_port_solution()
    zin_err = np.max(np.abs(_zin(sol.y) - _zin(g["y"])) / np.abs(_zin(g["y"])))
    assert zin_err <= 1e-6, zin_err
    assert rel_err(sol.y, g["y"]) < 1e-6
    assert s.last_refinement["iterations"] <= 4
