"""Cancellation and bounded device waits on the GPU.

Mirrors the reference's cancellation tests (``tests/test_cancel.py:82-247``):
a token raised before the solve aborts it even with the host checkpoints
silenced (the native factorisation polls the flag between panels, the
mixed solver also between refinement steps); a token tripped on the N-th
host checkpoint of a sweep aborts there; a token raised by another host
thread during a large factorisation aborts it; an untripped token leaves
results bit-identical; and an aborted solver solves again cleanly.

The bounded device waits are checked by making them run out on purpose
(``mw_selftest_wait_timeout``: a short limit and an event that never
comes); each must end with MW_ERR_TIMEOUT and leave the context usable.
"""

import ctypes as C
import threading
import time

import numpy as np
import pytest

from cases import CASES
from conftest import golden, rel_err

import momwire_b200
from momwire_b200 import CancelToken, SolveAborted, _lib
from momwire_b200.workloads import dipole_array

pytestmark = pytest.mark.gpu


def _trip_on_nth_checkpoint(solver, token, n):
    calls = [0]
    real = solver._checkpoint

    def counting():
        calls[0] += 1
        if calls[0] == n:
            token.cancel()
        real()

    solver._checkpoint = counting
    return calls, real


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["config1", "d2_junction_port"])
def test_native_poll_aborts_without_host_checkpoints(cuda_device, precision, name):
    token = CancelToken()
    token.cancel()
    s = momwire_b200.BSplineSolver(**CASES[name](), precision=precision, cancel=token)
    s._checkpoint = lambda: None  # only the native polls remain
    with pytest.raises(SolveAborted):
        s.compute_port_solution()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cancel_on_nth_checkpoint_mid_sweep(cuda_device, precision):
    token = CancelToken()
    s = momwire_b200.BSplineSolver(**CASES["config1"](), precision=precision, cancel=token)
    ks = np.linspace(0.9 * s.k, 1.1 * s.k, 12)
    calls, _ = _trip_on_nth_checkpoint(s, token, n=5)
    with pytest.raises(SolveAborted):
        s.compute_impedance_swept(ks)
    assert calls[0] == 5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["config1", "d2_junction_port", "d2_refl_normal"])
def test_untripped_token_is_bit_identical(cuda_device, precision, name):
    y_none = momwire_b200.BSplineSolver(**CASES[name](), precision=precision).compute_port_solution().y
    y_tok = momwire_b200.BSplineSolver(**CASES[name](), precision=precision,
                                       cancel=CancelToken()).compute_port_solution().y
    assert np.array_equal(y_none, y_tok)


def test_abort_leaves_no_residue(cuda_device):
    g = golden("d2_junction_port")
    token = CancelToken()
    s = momwire_b200.BSplineSolver(**CASES["d2_junction_port"](), cancel=token)
    _, real = _trip_on_nth_checkpoint(s, token, n=1)
    with pytest.raises(SolveAborted):
        s.compute_port_solution()
    s._cancel = None
    s._checkpoint = real
    assert rel_err(s.compute_port_solution().y, g["y"]) < 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_thread_cancel_during_large_factorisation(cuda_device, precision):
    """A host thread raises the token while the 16x16 array (10,496
    unknowns) is being factorised; the solve ends with SolveAborted well
    before a full solve would, and the solver then solves cleanly."""
    import torch

    kw = dipole_array(16, 16)
    token = CancelToken()
    s = momwire_b200.BSplineSolver(**kw, precision=precision, cancel=token)
    s.compute_port_solution()  # warm: tables, workspace, kernels
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s._cancel = None
    s.compute_port_solution()
    full = time.perf_counter() - t0
    s._cancel = token
    # the host enqueues the whole factorisation in a few ms; the fill has
    # to finish first, so a trip 2 ms after the call lands inside it
    timer = threading.Timer(0.002, token.cancel)
    t0 = time.perf_counter()
    timer.start()
    with pytest.raises(SolveAborted):
        s.compute_port_solution()
    aborted = time.perf_counter() - t0
    timer.join()
    torch.cuda.synchronize()
    assert aborted < full + 0.5
    s._cancel = None
    y = s.compute_port_solution().y
    assert rel_err(y, golden("array16x16")["y"]) < (1e-10 if precision == "fp64" else 1e-6)


@pytest.mark.parametrize("which", [0, 1], ids=["grid_barrier", "mbarrier"])
def test_bounded_wait_times_out_and_context_survives(cuda_device, which):
    import torch

    lib = _lib.load()
    ws = torch.zeros(16, dtype=torch.uint8, device=cuda_device)
    stream = torch.cuda.current_stream(cuda_device).cuda_stream
    t0 = time.perf_counter()
    st = lib.mw_selftest_wait_timeout(which, 1 << 16, C.c_void_p(ws.data_ptr()), C.c_void_p(stream))
    dt = time.perf_counter() - t0
    assert st == _lib.MW_ERR_TIMEOUT, lib.mw_last_error()
    assert b"gave up" in lib.mw_last_error()
    assert dt < 30.0
    # the context is still usable: a full solve right after
    y = momwire_b200.BSplineSolver(**CASES["config1"]()).compute_port_solution().y
    assert rel_err(y, golden("config1")["y"]) < 1e-10


def test_selftest_rejects_bad_arguments():
    lib = _lib.load()
    assert lib.mw_selftest_wait_timeout(2, 1 << 16, None, None) == _lib.MW_ERR_INVALID
    assert lib.mw_selftest_wait_timeout(0, 1 << 30, None, None) == _lib.MW_ERR_INVALID
    assert lib.mw_selftest_wait_timeout(0, 1 << 16, None, None) == _lib.MW_ERR_INVALID
