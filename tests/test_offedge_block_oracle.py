"""The block-sampler oracle pinned to the reference (CPU): seven blocks the
reference's own ``bspline_assemble_offedge_block`` family returned
(``tests/golden/make_offedge_blocks.py``) -- free space at degrees 1 and 2,
the PEC and reflection-coefficient images, the extended kernel with and
without the reflection-coefficient ground."""

import numpy as np
import pytest

from blocks import CASES, case
from conftest import rel_err
from oracle import block_oracle as BO


@pytest.mark.parametrize("name", CASES)
def test_oracle_block_matches_reference(name):
    a, want = case(name)
    got = BO.offedge_block(a["supp_I"], a["polys_I"], a["segl_I"], a["segr_I"], a["tan_I"], a["supp_J"],
                           a["polys_J"], a["segl_J"], a["segr_J"], a["tan_J"], a["a2"], a["k"], a["omega"],
                           a["eps_"], a["mu_"], a["t"], a["w"], group=a["group"], a_ek=a["a_ek"], refl=a["refl"])
    assert got.shape == want.shape
    assert rel_err(got, want) < 1e-12


def test_fixture_covers_the_variants():
    kinds = {n: case(n)[0] for n in CASES}
    assert any(k["refl"] is not None and k["group"] is not None for k in kinds.values())
    assert any(k["refl"] is None and k["group"] is not None for k in kinds.values())
    assert {k["degree"] for k in kinds.values()} == {1, 2}
