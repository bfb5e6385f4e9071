"""Cooperative cancellation, host side (no GPU needed).

The reference threads a ``CancelToken`` into its solvers through ``cancel=``
and polls it at phase boundaries; a raised token surfaces as
``SolveAborted`` (``_cancel.py:24-79``, ``tests/test_cancel.py:82-247``).
Here the token is polled by the host at the same seams and its flag address
is handed to the native factorisation, which polls it between panels.  These
tests need no device: a token raised before the solve must abort before any
device work starts.
"""

import numpy as np
import pytest

from cases import CASES

import momwire_b200
from momwire_b200 import CancelToken, SolveAborted


def _solver(name="config1", **extra):
    return momwire_b200.BSplineSolver(**CASES[name](), **extra)


def test_token_surface():
    t = CancelToken()
    assert not t.cancelled
    t.raise_if_cancelled()
    t.cancel()
    assert t.cancelled
    with pytest.raises(SolveAborted):
        t.raise_if_cancelled()
    # the native side reads an int32 at this address
    import ctypes

    assert isinstance(t.ptr, int) and t.ptr != 0
    assert ctypes.c_int32.from_address(t.ptr).value == 1


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize(
    "call",
    [
        lambda s: s.compute_port_solution(),
        lambda s: s.compute_y_matrix(),
        lambda s: s.compute_impedance(),
        lambda s: s.compute_y_matrix_swept(np.array([s.k, 1.01 * s.k])),
        lambda s: s.compute_impedance_swept(np.array([s.k])),
        lambda s: s.compute_port_solution_swept(np.array([s.k])),
    ],
    ids=["port_solution", "y_matrix", "impedance", "y_swept", "impedance_swept", "port_solution_swept"],
)
def test_precancelled_token_aborts_before_device_work(precision, call):
    token = CancelToken()
    token.cancel()
    s = _solver(precision=precision, cancel=token)
    with pytest.raises(SolveAborted):
        call(s)


def test_precancelled_junction_structure_aborts():
    token = CancelToken()
    token.cancel()
    s = _solver("d2_junction_port", cancel=token)
    with pytest.raises(SolveAborted):
        s.compute_port_solution()


def test_token_is_not_consumed_by_construction():
    # building the solver and its host tables never polls the token
    token = CancelToken()
    token.cancel()
    s = _solver("d2_junction_port", cancel=token)
    assert s._basis().n > 0
    assert s._geometry().n > 0
    assert token.cancelled
