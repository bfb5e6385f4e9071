"""Invalid inputs are refused as the reference refuses them: the same
exception type and text (recorded by ``tests/golden/make_refusals.py``),
at construction -- or at the solve, for the quadrature order -- and the
inputs the reference's constructor accepts are accepted."""

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
