"""The oracle (CPU restatement) pinned against the reference: its own
known-answer tests and golden vectors produced by running the reference."""

import numpy as np
import pytest

from cases import CASES, HD
from conftest import golden, rel_err
from oracle import bspline_oracle as O

# Known answers from the reference's tests/test_tent_parity.py:43-109
# (degree-1 pins, 1e-6 relative).
PINS = [
    (dict(wires=[np.array([[0.0, 0.0, -5.29], [0.0, 0.0, 5.29]])], nsegs=20, degree=1), 69.069365 - 20.348461j),
    (dict(wires=[np.array([[0.0, 0.0, -5.29], [0.0, 0.0, 5.29]])], nsegs=40, degree=1), 69.403082 - 19.237949j),
    (dict(wires=[np.array([[0.0, 0.0, -2.65], [0.0, 0.0, 2.65]])], nsegs=20, degree=1), 11.984894 - 942.538771j),
    (dict(wires=[np.array([[0.0, 0.0, -HD], [0.0, 0.0, HD]]),
                 np.array([[-2.2, 0.0, -1.05 * HD], [-2.2, 0.0, 1.05 * HD]])], nsegs=20, degree=1),
     27.793081 + 2.327531j),
    (dict(wires=[np.array([[-HD * np.cos(np.pi / 6), 0.0, HD * 0.5], [0.0, 0.0, 0.0],
                           [HD * np.cos(np.pi / 6), 0.0, HD * 0.5]])], nsegs=10, degree=1), 53.636373 - 32.936517j),
    (dict(wires=[np.array([[-HD, 0.0, 7.0], [HD, 0.0, 7.0]])], nsegs=20, degree=1, ground_z=0.0),
     93.328701 - 12.162851j),
]


@pytest.mark.parametrize("kw,z_pin", PINS)
def test_oracle_tent_pins(kw, z_pin):
    Y, *_ = O.port_solution(O.make_spec(**kw))
    z = 1.0 / Y[0, 0]
    assert abs(z - z_pin) <= 1e-6 * abs(z_pin), (z, z_pin)


def test_oracle_multifeed_pin():
    """test_tent_parity.py:93-103: two-port Y pins and reciprocity."""
    Y, *_ = O.port_solution(O.make_spec(**CASES["d1_multifeed"]()))
    assert abs(Y[0, 0] - (0.02086267 + 0.02461764j)) < 1e-7
    assert abs(Y[0, 1] - (-0.01344524 - 0.02291742j)) < 1e-7
    assert abs(Y[0, 1] - Y[1, 0]) < 1e-10


def test_oracle_config1_known_answer():
    """Config 1 driving-point impedance produced by the reference here."""
    Y, *_ = O.port_solution(O.make_spec(**CASES["config1"]()))
    z = 1.0 / Y[0, 0]
    assert abs(z - (67.5789431392556 - 30.968698608555457j)) <= 1e-9 * abs(z)


SMALL = [n for n in CASES if n != "array4x4"]


@pytest.mark.parametrize("name", SMALL)
def test_oracle_matches_reference_golden(name):
    g = golden(name)
    Y, X, Z, geom, basis = O.port_solution(O.make_spec(**CASES[name]()))
    assert rel_err(Z, g["Z"]) < 1e-10
    assert rel_err(Y, g["y"]) < 1e-10
    assert rel_err(X, g["coeffs"]) < 1e-9
    cur = np.concatenate(O.currents_at_knots(O.make_spec(**CASES[name]()), geom, basis, X[:, 0]))
    assert rel_err(cur, g["currents0"]) < 1e-9


def test_oracle_same_edge_static_converged():
    """The graded-panel static table is converged (20 vs 32 nodes)."""
    a = O.same_edge_static_table(0.0117, 0.0005, 41, 2, n_gl=20)
    b = O.same_edge_static_table(0.0117, 0.0005, 41, 2, n_gl=32)
    assert rel_err(a, b) < 1e-14
    a = O.same_edge_static_table(0.0117, 0.0005, 41, 2, ek=True, n_gl=20)
    b = O.same_edge_static_table(0.0117, 0.0005, 41, 2, ek=True, n_gl=32)
    assert rel_err(a, b) < 1e-14
