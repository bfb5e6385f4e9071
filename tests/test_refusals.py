"""Invalid inputs are refused as the reference refuses them: the same
exception type and text (recorded by ``tests/golden/make_refusals.py``),
at construction -- or at the solve, for the quadrature order -- and the
inputs the reference's constructor accepts are accepted.  Empty sweeps
return the reference's layouts without solving."""

import json
from pathlib import Path

import pytest

from refusal_cases import AT_SOLVE, REFUSALS

import momwire_b200

WANT = json.loads((Path(__file__).resolve().parent / "golden" / "refusals.json").read_text())


@pytest.mark.parametrize("name", sorted(REFUSALS))
def test_refusal_matches_reference(name):
    want = WANT[name]
    if want is None:
        momwire_b200.BSplineSolver(**REFUSALS[name]())
        return
    with pytest.raises(Exception) as err:
        s = momwire_b200.BSplineSolver(**REFUSALS[name]())
        if name in AT_SOLVE:
            s._dev_tables()  # the first use of the quadrature order
    assert type(err.value).__name__ == want["type"]
    assert str(err.value) == want["message"]


@pytest.mark.parametrize("name,shape", [("config1", (0,)), ("d1_yagi", (0,)), ("d2_junction_port", (0, 2))])
def test_empty_sweeps_have_the_reference_layout(name, shape):
    """An empty sweep solves nothing and returns the reference's layout
    (its shapes and dtypes, recorded from it for these cases)."""
    import numpy as np
    from cases import CASES

    s = momwire_b200.BSplineSolver(**CASES[name]())
    z = s.compute_impedance_swept(np.array([]))
    assert z.shape == shape and z.dtype == np.complex128
    n_p = 2 if name == "d2_junction_port" else 1
    y = s.compute_y_matrix_swept(np.array([]))
    assert y.shape == (0, n_p, n_p) and y.dtype == np.complex128
    assert s.compute_port_solution_swept(np.array([])) == []
