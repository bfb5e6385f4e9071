"""NEC-2 decks through the reference's deck front end, solved here: the
keywords its ``deck.build_solver`` passed to ``BSplineSolver`` give the
reference's Y on the GPU (FP64 path) and its port impedances within 1e-6
(mixed path)."""

import numpy as np
import pytest

from conftest import golden, rel_err
from decks import DECKS, deck_kwargs

import momwire_b200

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(DECKS))
def test_deck_solve_matches_reference(name, cuda_device):
    g = golden(f"deck_{name}")
    y = momwire_b200.BSplineSolver(**deck_kwargs(name)).compute_port_solution().y
    assert rel_err(y, g["y"]) < 1e-9


@pytest.mark.parametrize("name", sorted(DECKS))
def test_deck_solve_mixed_precision(name, cuda_device):
    g = golden(f"deck_{name}")
    y = momwire_b200.BSplineSolver(**deck_kwargs(name), precision="mixed").compute_port_solution().y
    zin = 1.0 / np.diag(y)
    assert np.max(np.abs(zin - g["zin"]) / np.abs(g["zin"])) <= 1e-6
