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


def _cgetrf(A, nrhs_max, device):
    import torch

    n = A.shape[0]
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).to(device)
    lib = _lib.load()
    wsb = lib.mw_cgetrf_workspace_size(n, nrhs_max)
    ws = torch.empty(wsb, dtype=torch.uint8, device=device)
    ipiv = torch.empty(n, dtype=torch.int32, device=device)
    info = torch.zeros(2, dtype=torch.int32, device=device)
    _lib.call("mw_cgetrf", n, Ad.data_ptr(), n, ipiv.data_ptr(), info.data_ptr(), ws.data_ptr(), wsb, nrhs_max, None,
              None)
    return Ad, ipiv, info, ws, wsb


@pytest.mark.parametrize("n,nrhs", [(390, 37), (1000, 300)])
def test_cgetrs_many_right_hand_sides(n, nrhs, cuda_device):
    """Triangular sweeps over several leaf CTAs, a partial last block and
    the fused next-block update (every leaf after the first)."""
    import torch

    rng = np.random.default_rng(7 * n + nrhs)
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    A += np.eye(n, dtype=np.complex64) * 2
    B = (rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))).astype(np.complex64)
    Ad, ipiv, info, ws, wsb = _cgetrf(A, nrhs, cuda_device)
    Bd = torch.from_numpy(np.ascontiguousarray(B.T)).to(cuda_device)
    _lib.call("mw_cgetrs", n, nrhs, Ad.data_ptr(), n, ipiv.data_ptr(), Bd.data_ptr(), n, ws.data_ptr(), wsb, None)
    inf = info.cpu().numpy()
    assert inf[0] == 0 and inf[1] == 0
    X = Bd.cpu().numpy().T.astype(np.complex128)
    want = scipy.linalg.solve(A.astype(np.complex128), B.astype(np.complex128))
    cond = np.linalg.cond(A.astype(np.complex128))
    assert rel_err(X, want) < 50 * cond * 6e-8


def test_cgetrf_exact_zero_pivot_reports_info(cuda_device):
    """LAPACK's convention on the complex64 panel: the 1-based column of
    the first exact zero pivot, no interchange and no scaling there."""
    n = 200
    A = np.eye(n, dtype=np.complex64)
    A[165, 165] = 0.0
    _Ad, ipiv, info, _ws, _wsb = _cgetrf(A, 1, cuda_device)
    assert info.cpu().numpy()[0] == 166
    assert np.array_equal(ipiv.cpu().numpy(), np.arange(1, n + 1))


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
    assert s.last_refinement["last_correction"] <= s.mixed_tol


@pytest.mark.parametrize("name", ["d1_dipole20", "d2_pec", "d2_ek_monopole_pec"])
def test_batched_fill_matches_single_fill(name, cuda_device):
    """Each matrix of one batched fill equals the single fill at its k, and
    its complex64 copy is the rounded complex128 matrix."""
    import torch

    s = momwire_b200.BSplineSolver(**CASES[name]())
    ks = np.array([0.8, 1.0, 1.25]) * s.k
    Z, Z32 = s._fill_batched(ks, torch.cuda.current_stream().cuda_stream)
    Zh, Z32h = Z.cpu().numpy(), Z32.cpu().numpy()
    for i, kk in enumerate(ks):
        with s._k_restored():
            s._set_k(kk)
            want = s._compute_Z_operator()
        assert rel_err(Zh[i].T, want) < 1e-13
        assert np.array_equal(Z32h[i], Zh[i].astype(np.complex64))


@pytest.mark.parametrize("name", ["d1_dipole20", "config1", "d2_pec", "d2_ek", "d2_ek_monopole_pec"])
def test_batched_sweep_matches_fp64_per_k(name, cuda_device):
    """The batched mixed sweep (one batched fill, one batched LU, FP64
    refinement) against per-frequency complex128 solves."""
    kw = CASES[name]()
    s64 = momwire_b200.BSplineSolver(**kw)
    ks = np.linspace(0.9, 1.1, 5) * s64.k
    y64 = s64.compute_y_matrix_swept(ks)
    smx = momwire_b200.BSplineSolver(**kw, precision="mixed")
    assert smx._swept_batched_available()
    ymx = smx.compute_y_matrix_swept(ks)
    for i in range(len(ks)):
        z64, zmx = _zin(y64[i]), _zin(ymx[i])
        assert np.max(np.abs(zmx - z64) / np.abs(z64)) <= 1e-6
    assert smx.k == s64.k


def test_batched_sweep_yagi_64_frequencies(cuda_device):
    """One seeded Yagi of the 512-structure sweep workload at its 64
    frequencies (25.2-30.8 MHz)."""
    from momwire_b200.workloads import yagi_sweep

    structs, ks = yagi_sweep(n_structures=3, n_freq=64, seed=0)
    kw = structs[2]
    y64 = momwire_b200.BSplineSolver(**kw).compute_y_matrix_swept(ks[::8])
    smx = momwire_b200.BSplineSolver(**kw, precision="mixed")
    ymx = smx.compute_y_matrix_swept(ks)
    z64 = 1.0 / y64[:, 0, 0]
    zmx = 1.0 / ymx[::8, 0, 0]
    assert np.max(np.abs(zmx - z64) / np.abs(z64)) <= 1e-6
    assert smx.last_refinement["iterations"] <= 5


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


@pytest.mark.parametrize("width", [8, 16, 32])
def test_batched_sweep_panel_widths(width, cuda_device):
    """Every panel width the autotuner may pick gives the same sweep."""
    kw = CASES["d2_pec"]()
    s64 = momwire_b200.BSplineSolver(**kw)
    ks = np.linspace(0.9, 1.1, 5) * s64.k
    y64 = s64.compute_y_matrix_swept(ks)
    smx = momwire_b200.BSplineSolver(**kw, precision="mixed")
    smx._panel_width = width
    ymx = smx.compute_y_matrix_swept(ks)
    for i in range(len(ks)):
        z64, zmx = _zin(y64[i]), _zin(ymx[i])
        assert np.max(np.abs(zmx - z64) / np.abs(z64)) <= 1e-6


def test_grouped_sweep_matches_per_structure(cuda_device):
    """Structures of different orders, port counts, grounds and loading in
    padded groups against each structure's own complex128 per-k solves."""
    from momwire_b200 import sweep
    from momwire_b200.workloads import yagi_sweep

    structs, ks = yagi_sweep(n_structures=4, n_freq=6, seed=3)
    structs = structs + [CASES["d1_multifeed"](), CASES["d2_pec"](), CASES["d2_loaded_dipole"](),
                         CASES["d2_junction_port"]()]
    kss = np.linspace(0.95, 1.05, 6)
    out = {}
    for i, kw in enumerate(structs):
        k0 = momwire_b200.BSplineSolver(**kw).k if i >= 4 else None
        out[i] = ks if k0 is None else kss * k0
    # one frequency list per call: group the Yagis, then the rest one by one
    got = sweep.grouped_mixed_sweep(structs, ks, indices=range(4))
    for i in range(4):
        y64 = momwire_b200.BSplineSolver(**structs[i]).compute_y_matrix_swept(ks)
        z64, zg = 1.0 / y64[:, 0, 0], 1.0 / got[i][:, 0, 0]
        assert np.max(np.abs(zg - z64) / np.abs(z64)) <= 1e-6
    for i in range(4, len(structs)):
        got = sweep.grouped_mixed_sweep(structs, out[i], indices=[i])
        y64 = momwire_b200.BSplineSolver(**structs[i]).compute_y_matrix_swept(out[i])
        for j in range(len(out[i])):
            z64, zg = _zin(y64[j]), _zin(got[i][j])
            assert np.max(np.abs(zg - z64) / np.abs(z64)) <= 1e-6


def test_grouped_sweep_shares_one_factorisation(cuda_device):
    """Two structures of different orders in one padded group give the same
    Y as each one batched alone."""
    from momwire_b200 import sweep
    from momwire_b200.workloads import yagi_sweep

    structs, ks = yagi_sweep(n_structures=12, n_freq=4, seed=5)
    ns = [momwire_b200.BSplineSolver(**kw)._basis().n for kw in structs]
    pairs = [(i, j) for i in range(12) for j in range(i + 1, 12)
             if ns[i] != ns[j] and sweep.padded_order(ns[i]) == sweep.padded_order(ns[j])]
    assert pairs, ns
    i, j = pairs[0]
    solvers = [momwire_b200.BSplineSolver(**structs[x], precision="mixed") for x in (i, j)]
    import torch

    st = torch.cuda.current_stream().cuda_stream
    nb = sweep.padded_order(ns[i])
    together, _ = sweep._solve_group(solvers, nb, ks, st, pw=16)
    for g, x in enumerate((i, j)):
        alone = momwire_b200.BSplineSolver(**structs[x], precision="mixed").compute_y_matrix_swept(ks)
        assert np.max(np.abs(together[g] - alone) / np.abs(alone)) <= 1e-6
