"""The learned Sommerfeld surrogate inside the fill: the fused tensor-core
remainder kernel against the oracle's Galerkin block with the same network,
whole solves against the quadrature-grid path, the domain fallback, and the
gain over the grid path on cold structures."""

import time

import numpy as np
import pytest

from cases import CASES
from conftest import rel_err
from oracle import bspline_oracle as O
from oracle import mlp_oracle as M
from oracle import sommerfeld_oracle as S

import momwire_b200
from momwire_b200 import _lib, surrogate, workloads

pytestmark = pytest.mark.gpu


class _NetGrid:
    """Duck-typed oracle grid whose surfaces come from the numpy MLP."""

    def __init__(self, params, lam, feats, factor):
        self.params, self.lam, self.feats, self.factor = params, lam, feats, factor
        self.r1_max = 4.0 * lam

    def eval(self, R1, theta):
        r1 = np.minimum(np.asarray(R1, dtype=float).ravel() / self.lam, 4.0)
        th = np.clip(np.asarray(theta, dtype=float).ravel(), 0.0, 0.5 * np.pi)
        X = np.empty((r1.size, 5), dtype=np.float32)
        X[:, 0] = (2.0 * np.sqrt(r1 / 4.0) - 1.0).astype(np.float32)
        X[:, 1] = (4.0 * th / np.pi - 1.0).astype(np.float32)
        X[:, 2:] = self.feats
        y = M.forward(X, self.params) * surrogate.SCALE * self.factor
        return (y[:, 0::2] + 1j * y[:, 1::2]).T


def test_fused_surrogate_q_matches_oracle(cuda_device):
    import torch

    kw = CASES["d2_somm_radials"]()
    s = momwire_b200.BSplineSolver(**kw)
    params = (M.init_params(21) * 0.4).astype(np.float32)
    model = surrogate.Surrogate(params, cuda_device)
    dt = s._dev_tables()
    n = s._basis().n
    Z = torch.zeros((n, n), dtype=torch.complex128, device=cuda_device)
    et = complex(O.eps_tilde(kw["ground_eps"], s.omega))
    f = s.omega / (2 * np.pi)
    feats = np.ascontiguousarray(surrogate.features(0.0, 1.0, et, f)[2:5], dtype=np.float32)
    factor = (s.omega * s.mu) / (surrogate.OMEGA_REF * surrogate.MU0_GRID)
    st = torch.cuda.current_stream().cuda_stream
    _lib.call("mw_somm_remainder_q_mlp", dt.seg, dt.basis, model.pbf.data_ptr(), model.p32.data_ptr(),
              feats.ctypes.data, float(s.wavelength), float(surrogate.SCALE * factor), 3, 0.0, float(s.k),
              Z.data_ptr(), n, None, n, model.err.data_ptr(), st)
    got = -Z.cpu().numpy().T
    assert int(model.err.item()) == 0
    spec = O.make_spec(**kw)
    geom = O.build_geometry(spec)
    basis = O.build_basis(spec, geom)
    want = S.remainder_Q(geom, basis.supp_seg, basis.polys, 2, 3, 0.0, spec.k,
                         _NetGrid(params, s.wavelength, feats, factor))
    assert rel_err(got, want) < 2e-4


def _weights():
    if not surrogate.WEIGHTS_PATH.exists():
        pytest.skip("no trained surrogate weights shipped")


def test_surrogate_solves_track_the_grid_path(cuda_device):
    """As an approximation (surrogate_tol=APPROX_TOL) the surrogate serves
    and stays within ZIN_TOL of the grid path."""
    _weights()
    structs = workloads.somm_structures(12, seed=7)
    errs = []
    for kw in structs:
        zg = momwire_b200.BSplineSolver(**kw).compute_impedance()[0]
        s = momwire_b200.BSplineSolver(**kw, sommerfeld_method="surrogate", surrogate_tol=surrogate.APPROX_TOL)
        zs = s.compute_impedance()[0]
        assert s.last_sommerfeld["method"] == "surrogate", s.last_sommerfeld
        errs.append(abs(zs - zg) / abs(zg))
    print("surrogate |dZin|/|Zin|:", ["%.2e" % e for e in errs])
    assert max(errs) <= surrogate.ZIN_TOL, errs


def test_surrogate_falls_back_outside_its_domain(cuda_device):
    _weights()
    kw = CASES["d2_somm_far_pair"]()  # 4.5 wavelengths apart: R1 > 4 lambda
    s = momwire_b200.BSplineSolver(**kw, sommerfeld_method="surrogate")
    y = s.compute_port_solution().y
    assert s.last_sommerfeld["method"] == "grid"
    assert "domain" in s.last_sommerfeld["reason"]
    y_grid = momwire_b200.BSplineSolver(**kw).compute_port_solution().y
    assert rel_err(y, y_grid) < 1e-14


def test_surrogate_gain_over_cold_grid(cuda_device):
    """Structures with their own ground and frequency each need a fresh
    grid master on the quadrature path; the surrogate needs none."""
    import torch

    from momwire_b200 import sommerfeld as P

    _weights()
    structs = workloads.somm_structures(24, seed=11)
    for method in ("grid", "surrogate"):  # warm-up (library load, kernels)
        momwire_b200.BSplineSolver(**structs[0], sommerfeld_method=method,
                                   surrogate_tol=surrogate.APPROX_TOL).compute_impedance()
    times = {}
    for method in ("grid", "surrogate"):
        P.clear_cache()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for kw in structs:
            momwire_b200.BSplineSolver(**kw, sommerfeld_method=method,
                                       surrogate_tol=surrogate.APPROX_TOL).compute_impedance()
        torch.cuda.synchronize()
        times[method] = time.perf_counter() - t0
    print("cold structures: grid %.3f s, surrogate %.3f s" % (times["grid"], times["surrogate"]))
    assert times["surrogate"] < times["grid"]


def test_surrogate_tolerance_is_validated():
    with pytest.raises(ValueError, match="surrogate_tol"):
        momwire_b200.BSplineSolver(**CASES["d2_somm_radials"](), sommerfeld_method="surrogate", surrogate_tol=0.0)


def test_sommerfeld_population_at_the_mixed_gate(cuda_device):
    """All 256 seeded Sommerfeld-ground structures (dipoles, monopoles with
    radials, inverted Vs over random grounds, 3-30 MHz): at the default
    surrogate_tol (1e-6) every structure the surrogate serves must be within
    1e-6 of the quadrature-grid path, and the fallback must fire for those
    whose spot check misses it; as an approximation (APPROX_TOL) the
    per-structure errors are stated and held to ZIN_TOL."""
    _weights()
    structs = workloads.somm_structures(256, seed=0)
    fell_back, approx, served = 0, [], 0
    for i, kw in enumerate(structs):
        zg = momwire_b200.BSplineSolver(**kw).compute_impedance()[0]
        s = momwire_b200.BSplineSolver(**kw, sommerfeld_method="surrogate")
        zs = s.compute_impedance()[0]
        e = abs(zs - zg) / abs(zg)
        if s.last_sommerfeld["method"] == "surrogate":
            served += 1
            assert e <= 1e-6, (i, e, s.last_sommerfeld)
        else:
            fell_back += 1
            assert e <= 1e-12, (i, e)  # the fallback is the grid path itself
        sa = momwire_b200.BSplineSolver(**kw, sommerfeld_method="surrogate", surrogate_tol=surrogate.APPROX_TOL)
        za = sa.compute_impedance()[0]
        approx.append((i, sa.last_sommerfeld["method"], abs(za - zg) / abs(zg)))
    print(f"surrogate at surrogate_tol=1e-6: served {served} of {len(structs)}, fell back {fell_back}")
    print("approximation (surrogate_tol=%.0e), per structure |dZin|/|Zin|:" % surrogate.APPROX_TOL)
    for i, m, e in approx:
        print(f"  {i:3d} {m:9s} {e:.2e}")
    assert served + fell_back == len(structs)
    assert fell_back > 0
    assert max(e for _i, m, e in approx if m == "surrogate") <= surrogate.ZIN_TOL
