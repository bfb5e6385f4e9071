"""Host-side tables of momwire_b200 against the oracle's restatement:
geometry, basis support and polynomials, KCL rows, port columns, tiles."""

import numpy as np
import pytest

from cases import CASES
from oracle import bspline_oracle as O

import momwire_b200
from momwire_b200 import _tables as T


@pytest.mark.parametrize("name", sorted(CASES))
def test_tables_match_oracle(name):
    kw = CASES[name]()
    s = momwire_b200.BSplineSolver(**kw)
    sp = O.make_spec(**kw)
    og = O.build_geometry(sp)
    ob = O.build_basis(sp, og)
    g, b = s._geometry(), s._basis()
    assert np.array_equal(g.seg_l, og["seg_l"]) and np.array_equal(g.seg_r, og["seg_r"])
    np.testing.assert_allclose(g.tangents, og["tangents"], rtol=0, atol=1e-15)
    assert np.array_equal(np.where(b.supp < 0, 0, b.supp), ob.supp_seg)
    np.testing.assert_allclose(b.polys, ob.polys, rtol=1e-12, atol=1e-12 * np.abs(ob.polys).max())
    assert np.array_equal(b.kcl_A.toarray(), ob.kcl_A)
    B, kcl = s._port_columns()
    Bo, kclo = O.port_columns(sp, og, ob)
    np.testing.assert_allclose(B, Bo, rtol=1e-13, atol=1e-14)
    assert np.array_equal(kcl.toarray(), kclo)
    # the sparse port entries the device scatter uses rebuild the same B
    r, c, v, n_p = s._port_entries()
    Bs = np.zeros((b.n, n_p), dtype=np.complex128)
    np.add.at(Bs, (r, c), v)
    np.testing.assert_allclose(Bs, Bo, rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("name", sorted(CASES))
def test_tiles_cover_every_wing(name):
    s = momwire_b200.BSplineSolver(**CASES[name]())
    b = s._basis()
    t = T.build_tiles(b.supp)
    assert t.max_basis <= T.MAX_TILE_BASIS and t.max_seg <= T.MAX_TILE_SEG
    assert int(t.nb.sum()) == b.n
    for ti in range(len(t.first)):
        for m in range(t.first[ti], t.first[ti] + t.nb[ti]):
            for a in range(b.supp.shape[1]):
                if b.supp[m, a] < 0:
                    assert t.loc[m, a] == -1
                else:
                    assert t.seg[ti, t.loc[m, a]] == b.supp[m, a]


def _greedy_tiles(supp, max_basis, max_seg):
    """Plain set-based statement of the greedy tiling."""
    out, m = [], 0
    while m < supp.shape[0]:
        cur, cnt = set(), 0
        while m + cnt < supp.shape[0] and cnt < max_basis:
            s = {int(x) for x in supp[m + cnt] if x >= 0}
            if len(cur | s) > max_seg:
                break
            cur |= s
            cnt += 1
        out.append((m, cnt, sorted(cur)))
        m += cnt
    return out


@pytest.mark.parametrize("name", ["d1_dipole20", "d2_junction", "d2_mixed_radius_kink", "d2_somm_plate8"])
@pytest.mark.parametrize("limits", [(16, 24), (5, 7), (3, 4)])
def test_tiles_are_the_greedy_split(name, limits):
    b = momwire_b200.BSplineSolver(**CASES[name]())._basis()
    t = T.build_tiles(b.supp, *limits)
    want = _greedy_tiles(b.supp, *limits)
    assert len(want) == len(t.first)
    for ti, (f, c, segs) in enumerate(want):
        assert (t.first[ti], t.nb[ti], t.ns[ti]) == (f, c, len(segs))
        assert list(t.seg[ti, : len(segs)]) == segs


@pytest.mark.parametrize("name", ["d1_dipole20", "d2_junction", "d2_ek_monopole_pec", "d2_somm_plate8"])
def test_kept_index_and_point_values(name):
    """The per-wire kept-basis lists, their vectorised global index, and
    the batched point evaluation against ``basis_values``."""
    s = momwire_b200.BSplineSolver(**CASES[name]())
    g, b = s._geometry(), s._basis()
    d = b.degree
    m = 0
    for w in range(len(b.kept)):
        kept = b.kept[w]
        n_b = len(b.knots[w]) - d - 1
        assert [k[4] for k in kept] == list(range(m, m + len(kept)))
        gi = b.kept.global_index(np.full(n_b, w), np.arange(n_b))
        want = np.full(n_b, -1)
        for j, _k, _jn, _e, mg in kept:
            want[j] = mg
        assert np.array_equal(gi, want)
        m += len(kept)
    assert m == b.n
    rng = np.random.default_rng(3)
    ws = rng.integers(0, len(b.kept), 40)
    xs = np.array([rng.uniform(0, g.wire_arc[w][-1]) for w in ws])
    xs[:3] = [g.wire_arc[ws[0]][0], g.wire_arc[ws[1]][-1], g.wire_arc[ws[2]][1]]
    vals, first = T.point_values(b.knots, d, ws, xs)
    for i, (w, x) in enumerate(zip(ws, xs)):
        full = T.basis_values(b.knots[w], d, [x])[0]
        assert np.array_equal(full[first[i] : first[i] + d + 1], vals[i])
        assert np.count_nonzero(np.delete(full, np.arange(first[i], first[i] + d + 1))) == 0


@pytest.mark.parametrize("name", ["d1_dipole20", "d2_junction", "d2_mixed_radius_kink", "d2_somm_plate8"])
def test_point_values_at_every_knot(name):
    """The batched point evaluation at every knot of every wire -- the
    right-open span rule's ties -- against the full design matrix."""
    s = momwire_b200.BSplineSolver(**CASES[name]())
    g, b = s._geometry(), s._basis()
    d = b.degree
    ws = np.concatenate([np.full(len(a), w) for w, a in enumerate(g.wire_arc)])
    xs = np.concatenate(g.wire_arc)
    vals, first = T.point_values(b.knots, d, ws, xs)
    for i, (w, x) in enumerate(zip(ws, xs)):
        full = T.basis_values(b.knots[w], d, [x])[0]
        assert np.array_equal(full[first[i] : first[i] + d + 1], vals[i])


def test_ek_labels_match_oracle():
    kw = CASES["d2_ek_monopole_pec"]()
    s = momwire_b200.BSplineSolver(**kw)
    sp = O.make_spec(**kw)
    og = O.build_geometry(sp)
    lab, lab_img = s._ek()
    ol, oli = O.ek_labels(sp, og, True)
    assert np.array_equal(lab, ol) and np.array_equal(lab_img, oli)


def test_constructor_validation_messages():
    w = [np.array([[0, 0, 0.0], [0, 0, 1.0]])]
    with pytest.raises(ValueError, match="degree must be >= 1"):
        momwire_b200.BSplineSolver(wires=w, degree=0)
    with pytest.raises(NotImplementedError, match="degree > 2"):
        momwire_b200.BSplineSolver(wires=w, degree=3)
    with pytest.raises(ValueError, match="ground_eps requires ground_z"):
        momwire_b200.BSplineSolver(wires=w, ground_eps=(13, 0.005))
    with pytest.raises(ValueError, match="feeds\\[0\\]: wire_index 3 out of range"):
        momwire_b200.BSplineSolver(wires=w, feeds=[(3, None, 1.0)])
    with pytest.raises(ValueError, match="wire_radius entries must be positive"):
        momwire_b200.BSplineSolver(wires=w, wire_radius=-1.0)
    with pytest.raises(ValueError, match="junction_ports: junction index 0 out of range"):
        momwire_b200.BSplineSolver(wires=w, junction_ports=[0])
    with pytest.raises(NotImplementedError, match="ground plane"):
        momwire_b200.BSplineSolver(wires=w, ground_z=0.0, ground_eps=(13, 0.005))


@pytest.mark.parametrize("q,exc,msg", [(0, ValueError, "deg must be a positive integer"),
                                       (9, RuntimeError, "n_qp > 8 not supported")])
def test_pair_quadrature_order_refused_at_the_solve(q, exc, msg):
    """As the reference: any order is taken by the constructor; a solve with
    none, or with more than eight points per segment, is refused."""
    s = momwire_b200.BSplineSolver(wires=[np.array([[0, 0, -5.0], [0, 0, 5.0]])], nsegs=21, wavelength=21.0,
                                   n_qp_pair=q)
    with pytest.raises(exc, match=msg):
        s._dev_tables()


@pytest.mark.parametrize("name", sorted(CASES))
def test_basis_count_and_kcl_rows_without_building(name):
    s = momwire_b200.BSplineSolver(**CASES[name]())
    n = s._basis_count()
    left = s._kcl_rows_left()
    assert n == s._basis().n
    kcl, _pa, _pv = s._split_kcl_ports(s._basis().kcl_A)
    assert left == kcl.shape[0]


def test_native_tiles_edge_cases():
    """mw_build_tiles: empty input, one basis per tile, and a basis wider
    than a tile is rejected with a clear error."""
    from momwire_b200 import _lib

    t = T.build_tiles(np.zeros((0, 3), dtype=np.int32))
    assert t.first.size == 0 and t.loc.shape == (0, 3)
    supp = np.array([[0, 1, 2], [1, 2, 3], [5, -1, -1]], dtype=np.int32)
    t = T.build_tiles(supp, max_basis=1, max_seg=3)
    assert list(t.first) == [0, 1, 2] and list(t.nb) == [1, 1, 1] and list(t.ns) == [3, 3, 1]
    assert list(t.loc[2]) == [0, -1, -1] and list(t.seg[2, :1]) == [5]
    with pytest.raises(_lib.NativeError, match="touches more segments than a tile holds"):
        T.build_tiles(supp, max_basis=4, max_seg=2)
