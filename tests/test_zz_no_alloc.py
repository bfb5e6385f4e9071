"""mw_fill_z_noalloc: the fill for callers that cannot allocate device memory.

Hosts that own every device allocation themselves (a plugin given only its
input and output buffers, or a foreign-language binding with no route to
cudaMalloc) cannot hand mw_fill_z its scratch table.  mw_fill_z_noalloc keeps
that table in a fixed device array inside the library instead.  This test
calls it through the C ABI twice in a row, on two different structures, and
checks each Z against the ordinary two-call path with a caller-owned table.
The file sorts last so that a run stopping at the first failure has already
run every other test.
"""

import ctypes as C

import numpy as np
import pytest

from cases import CASES
from conftest import rel_err

import momwire_b200
from momwire_b200 import _lib

pytestmark = pytest.mark.gpu


def _z_both_ways(name, device):
    import torch

    s = momwire_b200.BSplineSolver(**CASES[name]())
    dt = s._dev_tables()
    n = s._basis().n
    d = s.degree
    fr = _lib.Freq(float(s.k), float(s.omega), float(s.eps), float(s.mu))
    ek = int(s.extended_kernel)
    # ordinary path: caller-owned table
    table = torch.empty((dt.table_rows, d + 1, d + 1), dtype=torch.complex128, device=device)
    z_ref = torch.empty((n, n), dtype=torch.complex128, device=device)
    _lib.call("mw_same_edge_table", C.byref(dt.edges), d, s.n_qp_pair, ek, float(s.k), table.data_ptr(), None)
    _lib.call("mw_fill_z", C.byref(dt.seg), C.byref(dt.basis), table.data_ptr(), C.byref(dt.edges), C.byref(fr),
              s.n_qp_pair, z_ref.data_ptr(), n, None, n, None)
    # no-allocation path
    z_na = torch.full((n, n), float("nan"), dtype=torch.complex128, device=device)
    _lib.call("mw_fill_z_noalloc", C.byref(dt.seg), C.byref(dt.basis), C.byref(dt.edges), C.byref(fr), s.n_qp_pair,
              ek, z_na.data_ptr(), n, None)
    torch.cuda.synchronize()
    return z_na.cpu().numpy(), z_ref.cpu().numpy()


def test_noalloc_fill_matches_allocating_fill_twice(cuda_device):
    # two calls in a row on different structures: the shared table keeps
    # the previous call's rows, which must not leak into the next result
    for name in ("array4x4", "d2_mixed_radius_kink"):
        z_na, z_ref = _z_both_ways(name, cuda_device)
        assert np.all(np.isfinite(z_na))
        assert rel_err(z_na, z_ref) < 1e-12


def test_noalloc_rejects_oversized_table(cuda_device):
    import torch

    lib = _lib.load()
    s = momwire_b200.BSplineSolver(**CASES["config1"]())
    dt = s._dev_tables()
    cap = lib.mw_fill_z_noalloc_capacity(s.degree)
    assert cap == 32768
    # 4.5 MiB of doubles: 8 per row at degree 1, 18 at degree 2; no other
    # degree is served
    assert lib.mw_fill_z_noalloc_capacity(1) == 73728
    assert [lib.mw_fill_z_noalloc_capacity(d) for d in (-1, 0, 3, 4)] == [0, 0, 0, 0]
    edges = _lib.Edges.from_buffer_copy(dt.edges)
    edges.table_rows = cap + 1  # rejected on the host, before any launch
    fr = _lib.Freq(float(s.k), float(s.omega), float(s.eps), float(s.mu))
    n = s._basis().n
    z = torch.zeros((n, n), dtype=torch.complex128, device=cuda_device)
    st = lib.mw_fill_z_noalloc(C.byref(dt.seg), C.byref(dt.basis), C.byref(edges), C.byref(fr), s.n_qp_pair, 0,
                               z.data_ptr(), n, None)
    assert st == _lib.MW_ERR_WORKSPACE
    assert b"scratch" in lib.mw_last_error()
    assert float(z.abs().max()) == 0.0
