"""The enrichment oracle pinned to the reference (CPU).

``tests/golden/make_enrich.py`` recorded, for twelve structures with K >= 3
junctions (and one K = 2 case at enrichment_min_k=2), the reference's
enrichment specs, its three enrichment blocks Z_pe, Z_ep, Z_ee (ground
reaction included: PEC, reflection-coefficient and Sommerfeld grounds) and
its augmented port solution for the raw, stable, tikhonov and auto
variants.  The oracle (``oracle/enrich_oracle.py``) must reproduce them."""

import numpy as np
import pytest

from cases import ENRICH_CASES
from conftest import golden, rel_err
from oracle import bspline_oracle as O
from oracle import enrich_oracle as EO

ENR_KEYS = ("use_singular_enrichment", "enrichment_variant", "enrichment_min_k", "tikhonov_lambda", "n_qp_sing",
            "auto_tap_ratio_threshold")


def split(name):
    kw = ENRICH_CASES[name]()
    ek = {k: kw.pop(k) for k in list(kw) if k in ENR_KEYS}
    return kw, ek


def master(g):
    if "somm_n_region" not in g:
        return None
    return [g[f"somm_vals_{i}"] for i in range(int(g["somm_n_region"]))]


@pytest.mark.parametrize("name", sorted(ENRICH_CASES))
def test_oracle_enrichment_matches_reference(name):
    kw, ek = split(name)
    g = golden(name)
    sp = O.make_spec(**kw)
    geom = O.build_geometry(sp)
    basis = O.build_basis(sp, geom)
    variant = ek.get("enrichment_variant", "raw")
    min_k = ek.get("enrichment_min_k", 3)
    active = None if g["auto_active"].tolist() == [-1] else g["auto_active"].tolist()
    specs = EO.specs(sp, geom, min_k, active)
    assert [s[3] for s in specs] == g["spec_seg"].tolist()
    assert [s[4] for s in specs] == g["spec_origin"].tolist()
    mv = master(g)
    if specs:
        grid = O.sommerfeld_grid(sp, geom, mv) if mv is not None else None
        blocks = EO.blocks(sp, geom, basis, specs, "stable" if variant == "stable" else "raw", somm_grid=grid)
        for got, key in zip(blocks, ("Z_pe", "Z_ep", "Z_ee")):
            assert rel_err(got, g[key]) < 1e-12, key
    Y, X, _ = EO.port_solution(sp, variant, min_k, tikhonov_lambda=ek.get("tikhonov_lambda", 1e-3),
                               somm_master_values=mv)
    assert rel_err(Y, g["y"]) < 1e-11
    assert rel_err(X, g["coeffs"]) < 1e-11


def test_projection_coefficients():
    """The stable variant's subtracted polynomial vanishes at both ends and
    leaves the remainder orthogonal to every bubble (degree 2 and 3)."""
    t, w = O.gl01(200)
    for d in (1, 2, 3):
        c = EO.projection_coeffs(d)
        p = np.polynomial.polynomial.polyval
        assert abs(p(0.0, c)) < 1e-15 and abs(p(1.0, c)) < 1e-14
        r = t * np.log(t) - p(t, c)
        for i in range(d - 1):
            assert abs(np.sum(w * r * (t ** (i + 1) - t ** (i + 2)))) < 1e-6
