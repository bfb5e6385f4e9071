"""The reference's NEC-2 deck corpus solved here: the keywords its deck
front end handed ``BSplineSolver`` for each of the 60 decks give the
reference's Y on the GPU (FP64 path, 1e-9 of the largest entry) and its port
impedances within 1e-6 (mixed path)."""

import numpy as np
import pytest

from conftest import rel_err
from decks import corpus_kwargs
from test_deck_corpus import SERVED

import momwire_b200

pytestmark = pytest.mark.gpu

_REF = np.load(__import__("pathlib").Path(__file__).resolve().parent / "golden" / "deck_corpus.npz")


@pytest.mark.parametrize("name", SERVED)
def test_corpus_solve_matches_reference(name, cuda_device):
    y = momwire_b200.BSplineSolver(**corpus_kwargs(name)).compute_port_solution().y
    assert rel_err(y, _REF[f"y_{name}"]) < 1e-9


@pytest.mark.parametrize("name", SERVED)
def test_corpus_solve_mixed_precision(name, cuda_device):
    y = momwire_b200.BSplineSolver(**corpus_kwargs(name), precision="mixed").compute_port_solution().y
    zin, want = 1.0 / np.diag(y), _REF[f"zin_{name}"]
    assert np.max(np.abs(zin - want) / np.abs(want)) <= 1e-6
