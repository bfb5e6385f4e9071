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
            # the host part of a solve: basis (end topology), port split,
            # then the first use of the quadrature order
            s._basis()
            s._port_entries()
            s._dev_tables()
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


def test_capabilities_declaration():
    """The class-level declaration consumers read (the reference's
    ``capabilities`` interface) with this package's values."""
    cap = momwire_b200.BSplineSolver.capabilities
    assert cap.grounds == frozenset({"pec", "refl-coef", "sommerfeld"})
    assert cap.wire_loading and cap.extended_kernel and cap.junction_ports and cap.node_gaps
    assert cap.per_wire_radius and cap.singular_enrichment
    assert cap.refusal("sommerfeld", "junction_ports") is None
    assert cap.refusal("wire_loading") is None
    assert cap.refusal("singular_enrichment") is None
    assert "distributed wire loading" in cap.refusal("wire_loading", "singular_enrichment")
    assert "extended_kernel=True" in cap.refusal("extended_kernel", "singular_enrichment")
    assert "per-wire radii" in cap.refusal("per_wire_radius", "singular_enrichment")
    assert "ground contact is refused" in cap.refusal("refl-coef", "contact")
    assert cap.refusal("bogus_axis") is None  # a condition token alone is served


def test_enrichment_settings_are_kept():
    from refusal_cases import REFUSALS

    s = momwire_b200.BSplineSolver(**REFUSALS["enrichment_settings_with_enrichment_off"]())
    assert (s.use_singular_enrichment, s.n_qp_sing, s.enrichment_min_k, s.enrichment_variant) == (False, 16, 4,
                                                                                                  "stable")
    assert (s.tikhonov_lambda, s.auto_tap_ratio_threshold) == (1e-2, 0.5)
