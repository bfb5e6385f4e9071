"""Host-side table builders for the B-spline dense path (all O(N)).

These produce the plain arrays the native library consumes: per-segment
geometry, per-edge descriptors for the same-edge analytic split, the basis
support map and monomial coefficients, the fill's basis tiles, the
extended-kernel coaxial labels and the port columns.  Each builder restates
the reference routine it cites (paths relative to momwire's ``src/momwire``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.sparse

MAX_TILE_BASIS = 16
MAX_TILE_SEG = 24


# ---------------------------------------------------------------------------
# geometry  (bspline.py:988-1093)
# ---------------------------------------------------------------------------


@dataclass
class Geometry:
    seg_l: np.ndarray  # (N, 3)
    seg_r: np.ndarray  # (N, 3)
    tangents: np.ndarray  # (N, 3)
    h: np.ndarray  # (N,)
    radius: np.ndarray  # (N,)
    edge: np.ndarray  # (N,) int32
    pos_in_edge: np.ndarray  # (N,) int32
    edge_first: np.ndarray  # (E,)
    edge_n: np.ndarray  # (E,)
    edge_h: np.ndarray  # (E,)
    edge_radius: np.ndarray  # (E,)
    wire_first: np.ndarray  # (W,)
    wire_n: np.ndarray  # (W,)
    wire_arc: list  # per wire (n_w+1,) arc length at knots

    @property
    def n(self) -> int:
        return int(self.seg_l.shape[0])


def build_geometry(wires, npe, radius_per_wire) -> Geometry:
    """Uniform segments on every polyline edge: knots by linspace between
    the edge's anchors, h = |edge| / n (``bspline.py:1027-1050``).  All
    edges of all wires are laid out in one pass."""
    n_pts = np.fromiter((len(pl) for pl in wires), dtype=np.int64, count=len(wires))
    pts = np.concatenate([np.asarray(pl, dtype=np.float64) for pl in wires], axis=0)
    # an edge starts at every point but a wire's last
    is_start = np.ones(pts.shape[0], dtype=bool)
    is_start[np.cumsum(n_pts) - 1] = False
    p0 = pts[is_start]
    p1 = pts[np.flatnonzero(is_start) + 1]
    e_n = np.concatenate([np.asarray(c, dtype=np.int64).reshape(-1) for c in npe])
    e_wire = np.repeat(np.arange(len(wires), dtype=np.int64), n_pts - 1)
    if e_n.shape[0] != p0.shape[0]:
        raise ValueError("one segment count per polyline edge is needed")
    vec = p1 - p0
    L = np.sqrt((vec[:, None, :] @ vec[:, :, None])[:, 0, 0])  # same dot as a per-edge norm
    if (L < 1e-15).any():
        e = int(np.argmax(L < 1e-15))
        w = int(e_wire[e])
        first_edge = int(np.argmax(e_wire == w))
        raise ValueError(f"wire {w} edge {e - first_edge} has zero length")
    E = e_n.shape[0]
    e_first = np.concatenate(([0], np.cumsum(e_n)[:-1]))
    N = int(e_n.sum())
    edge = np.repeat(np.arange(E), e_n)
    pos = np.arange(N) - e_first[edge]
    step = 1.0 / e_n[edge]
    tl = pos * step
    tr = np.where(pos + 1 == e_n[edge], 1.0, (pos + 1) * step)
    seg_l = (1 - tl)[:, None] * p0[edge] + tl[:, None] * p1[edge]
    seg_r = (1 - tr)[:, None] * p0[edge] + tr[:, None] * p1[edge]
    e_h = L / e_n
    radius_e = np.asarray([float(radius_per_wire[w]) for w in range(len(wires))], dtype=np.float64)[e_wire]
    h = e_h[edge]
    w_n = np.bincount(e_wire, weights=e_n, minlength=len(wires)).astype(np.int64)
    w_first = np.concatenate(([0], np.cumsum(w_n)[:-1])).astype(np.int64)
    # arc length at knots per wire: one row-wise running sum over a padded
    # table (the same left-to-right additions as a per-wire cumsum)
    pad = np.zeros((len(wires), int(w_n.max(initial=0)) + 1))
    col = np.arange(h.shape[0]) - np.repeat(w_first, w_n)
    pad[np.repeat(np.arange(len(wires)), w_n), col + 1] = h
    np.cumsum(pad[:, 1:], axis=1, out=pad[:, 1:])
    w_arc = [pad[w, : n + 1] for w, n in enumerate(w_n.tolist())]
    return Geometry(
        seg_l=np.ascontiguousarray(seg_l),
        seg_r=np.ascontiguousarray(seg_r),
        tangents=np.ascontiguousarray((vec / L[:, None])[edge]),
        h=h,
        radius=radius_e[edge],
        edge=edge.astype(np.int32),
        pos_in_edge=pos.astype(np.int32),
        edge_first=e_first.astype(np.int32),
        edge_n=e_n.astype(np.int32),
        edge_h=e_h,
        edge_radius=radius_e,
        wire_first=w_first,
        wire_n=w_n,
        wire_arc=w_arc,
    )


# ---------------------------------------------------------------------------
# B-spline basis  (bspline.py:1216-1414)
# ---------------------------------------------------------------------------


def _span_values(knots, d, span, x):
    """The d+1 B-splines active on knot span ``span`` evaluated at x, using
    that span's polynomial pieces (triangular Cox-de Boor recursion)."""
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    span = np.broadcast_to(np.asarray(span), x.shape)
    N = np.zeros(x.shape + (d + 1,))
    N[..., 0] = 1.0
    left = np.zeros(x.shape + (d + 1,))
    right = np.zeros(x.shape + (d + 1,))
    for j in range(1, d + 1):
        left[..., j] = x - knots[span + 1 - j]
        right[..., j] = knots[span + j] - x
        saved = np.zeros(x.shape)
        for r in range(j):
            tmp = N[..., r] / (right[..., r + 1] + left[..., j - r])
            N[..., r] = saved + right[..., r + 1] * tmp
            saved = left[..., j - r] * tmp
        N[..., j] = saved
    return N


def point_values(knots_list, d, wires, xs):
    """Values of the d+1 active bases at one point per entry (wire w_i, arc
    position x_i): (vals (n, d+1), first active local basis index (n,)).
    Same span rule as ``basis_values``; one batched Cox-de Boor evaluation
    over 2d-knot windows."""
    n = len(xs)
    xs = np.asarray(xs, dtype=np.float64).reshape(-1)
    w = np.asarray(wires, dtype=np.int64).reshape(-1)
    lens = np.fromiter((len(k) for k in knots_list), dtype=np.int64, count=len(knots_list))
    offs = np.concatenate(([0], np.cumsum(lens)[:-1])).astype(np.int64)
    cat = np.concatenate(knots_list) if len(knots_list) else np.zeros(0)
    # bisect-right of x in its own wire's knot vector, all points at once
    # (the index np.searchsorted(kn, x, side="right") returns)
    lo = offs[w].copy()
    hi = lo + lens[w]
    while True:
        act = lo < hi
        if not act.any():
            break
        mid = (lo + hi) // 2
        right = act & (cat[np.minimum(mid, cat.size - 1)] <= xs)
        left = act & ~right
        lo = np.where(right, mid + 1, lo)
        hi = np.where(left, mid, hi)
    n_b = lens[w] - d - 1
    sp = np.minimum(np.maximum(lo - offs[w] - 1, d), n_b - 1)
    K = cat[(offs[w] + sp + 1 - d)[:, None] + np.arange(2 * d)[None, :]].reshape(n, 2 * d)
    first = (sp - d).astype(np.int64)
    span = np.arange(n) * (2 * d) + (d - 1)
    vals = _span_values(K.ravel(), d, span, xs)
    return vals.reshape(n, d + 1), first


def basis_values(knots, d, x):
    """(len(x), n_basis) values of every basis of a clamped knot vector
    (right-open spans; the final knot belongs to the last non-empty span)."""
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    n_b = len(knots) - d - 1
    span = np.searchsorted(knots, x, side="right") - 1
    span = np.clip(span, d, n_b - 1)
    vals = _span_values(knots, d, span, x)
    out = np.zeros((x.size, n_b))
    rows = np.arange(x.size)
    for c in range(d + 1):
        out[rows, span - d + c] = vals[:, c]
    return out


class KeptBases:
    """Per wire, the list of kept bases as (j_local, kind, junction, end,
    m_global) tuples (kind "int" interior, "dir" held by a junction, "gnd"
    held by the ground), built on first access of a wire."""

    def __init__(self, ends, n_b, m_first):
        self._ends = ends
        self._n_b = [int(x) for x in n_b]
        self._m_first = [int(x) for x in m_first]
        self._cache = {}

    def __len__(self):
        return len(self._ends)

    def __getitem__(self, w):
        if w < 0:
            w += len(self)
        if not 0 <= w < len(self):
            raise IndexError(w)
        out = self._cache.get(w)
        if out is None:
            es, ee = self._ends[w]
            n_b, m = self._n_b[w], self._m_first[w]
            out = []
            if es is not None:
                out.append((0, es[0], es[1], "start", m))
            base = m + len(out) - 1
            out.extend((j, "int", None, None, base + j) for j in range(1, n_b - 1))
            if ee is not None:
                out.append((n_b - 1, ee[0], ee[1], "end", m + len(out)))
            self._cache[w] = out
        return out

    def __iter__(self):
        return (self[w] for w in range(len(self)))

    def global_index(self, w, j):
        """Global basis index of local basis j of wire w (arrays of equal
        shape); -1 where that basis is not kept (a free end)."""
        w = np.asarray(w, dtype=np.int64)
        j = np.asarray(j, dtype=np.int64)
        has_s = np.array([e[0] is not None for e in self._ends], dtype=np.int64)[w]
        has_e = np.array([e[1] is not None for e in self._ends], dtype=np.int64)[w]
        n_b = np.asarray(self._n_b, dtype=np.int64)[w]
        m = np.asarray(self._m_first, dtype=np.int64)[w] + j - 1 + has_s
        ok = ((j > 0) | (has_s == 1)) & ((j < n_b - 1) | (has_e == 1)) & (j >= 0) & (j < n_b)
        return np.where(ok, m, -1)

    def __eq__(self, other):
        return len(self) == len(other) and all(a == b for a, b in zip(self, other))


@dataclass
class Basis:
    degree: int
    supp: np.ndarray  # (n_b, d+1) int32, -1 = padded wing
    polys: np.ndarray  # (n_b, d+1, d+1)
    kcl_A: "scipy.sparse.csr_matrix"  # (n_c, n_b) KCL rows, entries +-1
    kcl_junction: np.ndarray  # (n_c,) int64: the junction of each KCL row (ascending)
    knots: list  # per wire
    kept: KeptBases  # per wire: list of (j_local, kind, junction, end, m_global)

    @property
    def n(self) -> int:
        return int(self.supp.shape[0])


def build_basis(geom: Geometry, degree, ends, n_junctions, grounded) -> Basis:
    """Clamped knot vector per wire; keep interior bases plus the value-1
    end basis at junction / ground ends (``ends``: the (n_wires, 2) table of
    end holders of ``_topology.end_table`` -- junction index, FREE or
    GROUND); one KCL row per junction off the ground, in junction order;
    per-wing monomial coefficients in
    local arc length from values at d+1 uniform points (the reference's
    design-matrix + Vandermonde step, ``bspline.py:1318-1414``), computed by
    the native host routine ``mw_basis_polys``: segment s of a wire reads the
    knots at spans s+1-d .. s+d, which in the clamped vector are the wire's
    arc positions at indices clip(s+t, 0, n_w) for t in 1-d .. d."""
    d = int(degree)
    n_wires = len(geom.wire_first)
    wire_n = np.asarray(geom.wire_n, dtype=np.int64)
    firsts = np.asarray(geom.wire_first, dtype=np.int64)
    arcs = geom.wire_arc
    knots_all = [np.concatenate([np.zeros(d), arc, np.full(d, arc[-1])]) for arc in arcs]
    # ---- kept bases: interior bases, plus end bases a junction / ground holds
    from ._topology import FREE, GROUND

    def end_kind(code):
        if code == GROUND:
            return ("gnd", None)
        if code == FREE:
            return None
        return ("dir", int(code))

    ends = [(end_kind(ends[w, 0]), end_kind(ends[w, 1])) for w in range(n_wires)]
    has_s = np.fromiter((e[0] is not None for e in ends), dtype=np.int64, count=n_wires)
    has_e = np.fromiter((e[1] is not None for e in ends), dtype=np.int64, count=n_wires)
    n_kept = (wire_n + d - 2) + has_s + has_e
    m_first = np.concatenate(([0], np.cumsum(n_kept)[:-1])).astype(np.int64)
    m = int(n_kept.sum())
    jdirs = {j: [] for j in range(n_junctions)}
    for w, (es, ee) in enumerate(ends):
        if es is not None and es[0] == "dir":
            jdirs[es[1]].append((int(m_first[w]), 1.0))
        if ee is not None and ee[0] == "dir":
            jdirs[ee[1]].append((int(m_first[w] + n_kept[w] - 1), -1.0))
    bw = np.repeat(np.arange(n_wires), n_kept)
    # local basis index: 1 - has_start at a wire's first kept basis, +1 after
    js = np.arange(m) - np.repeat(m_first, n_kept) + np.repeat(1 - has_s, n_kept)
    # supports and per-wing monomial coefficients: native host routine
    import ctypes as C

    from . import _lib

    garc = np.ascontiguousarray(np.concatenate(arcs), dtype=np.float64)
    arc_off = np.ascontiguousarray(np.concatenate(([0], np.cumsum(wire_n + 1)[:-1])), dtype=np.int64)
    js = np.ascontiguousarray(js, dtype=np.int64)
    bw = np.ascontiguousarray(bw, dtype=np.int64)
    supp = np.empty((m, d + 1), dtype=np.int32)
    poly = np.empty((m, d + 1, d + 1))
    _lib.call("mw_basis_polys", garc.ctypes.data, arc_off.ctypes.data, np.ascontiguousarray(wire_n).ctypes.data,
              np.ascontiguousarray(firsts).ctypes.data, n_wires, d, js.ctypes.data, bw.ctypes.data, m,
              supp.ctypes.data, poly.ctypes.data)
    rows = [j for j in range(n_junctions) if j not in grounded]
    ri, ci, vi = [], [], []
    for r, j in enumerate(rows):
        for mg, sg in jdirs[j]:
            ri.append(r)
            ci.append(mg)
            vi.append(sg)
    # sparse: a few +-1 per junction row (4,225 x 33,280 dense would be 1.1 GB)
    kcl = scipy.sparse.csr_matrix((np.asarray(vi, dtype=np.float64), (np.asarray(ri, dtype=np.int64),
                                   np.asarray(ci, dtype=np.int64))), shape=(len(rows), m))
    return Basis(
        degree=d,
        supp=supp,
        polys=poly,
        kcl_A=kcl,
        kcl_junction=np.asarray(rows, dtype=np.int64),
        knots=knots_all,
        kept=KeptBases(ends, wire_n + d, m_first),
    )


# ---------------------------------------------------------------------------
# fill tiles
# ---------------------------------------------------------------------------


@dataclass
class Tiles:
    first: np.ndarray  # (T,) int32
    nb: np.ndarray  # (T,) int32
    ns: np.ndarray  # (T,) int32
    seg: np.ndarray  # (T, max_seg) int32
    loc: np.ndarray  # (n_b, d+1) int32
    max_basis: int
    max_seg: int


def build_tiles(supp: np.ndarray, max_basis=MAX_TILE_BASIS, max_seg=MAX_TILE_SEG) -> Tiles:
    """Greedy split of the basis list into runs of consecutive bases whose
    wings touch at most ``max_seg`` distinct segments (native host routine
    ``mw_build_tiles``)."""
    import ctypes as C

    from . import _lib

    supp = np.ascontiguousarray(supp, dtype=np.int32)
    n_b, wings = supp.shape
    cap = max(n_b, 1)
    first = np.zeros(cap, dtype=np.int32)
    nb = np.zeros(cap, dtype=np.int32)
    ns = np.zeros(cap, dtype=np.int32)
    seg = np.full((cap, max_seg), -1, dtype=np.int32)
    loc = np.full((cap, wings), -1, dtype=np.int32)
    nt = C.c_int64(0)
    _lib.call("mw_build_tiles", supp.ctypes.data, n_b, wings, int(max_basis), int(max_seg), first.ctypes.data,
              nb.ctypes.data, ns.ctypes.data, seg.ctypes.data, loc.ctypes.data, C.byref(nt))
    T = int(nt.value)
    used = int(ns[:T].max()) if T else 1
    return Tiles(
        first=first[:T].copy(),
        nb=nb[:T].copy(),
        ns=ns[:T].copy(),
        seg=np.ascontiguousarray(seg[:T, :used]),
        loc=loc[:n_b].copy(),
        max_basis=int(nb[:T].max()) if T else 1,
        max_seg=used,
    )


def edge_table_offsets(edge_n: np.ndarray):
    """Row offset of each edge in the same-edge Toeplitz table."""
    rows = 2 * edge_n.astype(np.int64) - 1
    off = np.concatenate([[0], np.cumsum(rows)[:-1]]).astype(np.int64)
    return off, int(rows.sum())


# ---------------------------------------------------------------------------
# extended kernel labels  (_bspline_kernels.py:249-321, bspline.py:2040-2088)
# ---------------------------------------------------------------------------


def ek_axis_groups(seg_l, seg_r, tangents, seg_a, tol=1e-6):
    """Coaxial-and-equal-radius labels: a segment joins the first existing
    group whose representative is (anti)parallel within ``tol``, has the
    same radius within ``tol`` and whose axis passes within ``tol*a`` of
    the segment centre; otherwise it starts a new group."""
    centers = 0.5 * (seg_l + seg_r)
    n = seg_a.shape[0]
    labels = np.empty(n, dtype=np.int32)
    rc = np.empty((0, 3))
    rt = np.empty((0, 3))
    ra = np.empty(0)
    for i in range(n):
        if ra.size:
            col = np.abs(rt @ tangents[i]) >= 1.0 - tol
            same = np.abs(seg_a[i] / ra - 1.0) <= tol
            dv = centers[i][None, :] - rc
            ax = dv @ tangents[i]
            perp = dv - ax[:, None] * tangents[i][None, :]
            co = np.linalg.norm(perp, axis=1) <= tol * ra
            hit = np.flatnonzero(col & same & co)
            if hit.size:
                labels[i] = int(hit[0])
                continue
        labels[i] = ra.size
        rc = np.vstack([rc, centers[i]])
        rt = np.vstack([rt, tangents[i]])
        ra = np.append(ra, seg_a[i])
    return labels


def mirror_points(p, gz):
    """Reflect points through z = gz (``_ground_mirror.py:37``)."""
    q = np.array(p, dtype=np.float64, copy=True)
    q[..., 2] = 2.0 * gz - q[..., 2]
    return q


def ek_labels(geom: Geometry, ground_z=None):
    """(labels, image labels): the real segments' labels, and for a ground
    plane the labels of the mirrored sources from one joint scan."""
    lab = ek_axis_groups(geom.seg_l, geom.seg_r, geom.tangents, geom.radius)
    if ground_z is None:
        return lab, None
    n = geom.n
    joint = ek_axis_groups(
        np.vstack([geom.seg_l, mirror_points(geom.seg_l, ground_z)]),
        np.vstack([geom.seg_r, mirror_points(geom.seg_r, ground_z)]),
        np.vstack([geom.tangents, geom.tangents * np.array([1.0, 1.0, -1.0])]),
        np.concatenate([geom.radius, geom.radius]),
    )
    return joint[:n].astype(np.int32), joint[n:].astype(np.int32)


def eps_tilde(ground_eps, omega, eps0):
    """Complex relative permittivity (``_ground_refl.py:46-60``)."""
    if isinstance(ground_eps, (tuple, list)):
        if len(ground_eps) != 2:
            raise ValueError(f"ground_eps tuple must be (eps_r, sigma), got {ground_eps!r}")
        er, sig = ground_eps
        return complex(float(er), -float(sig) / (omega * eps0))
    return complex(ground_eps)


def touch_tol(polyline) -> float:
    """Ground-contact snap distance: 1e-6 of the polyline length
    (``_ground_spec.py:127-153``)."""
    pl = np.asarray(polyline, dtype=np.float64)
    length = float(np.sum(np.linalg.norm(np.diff(pl, axis=0), axis=1)))
    return 1e-6 * max(length, 1e-30)


def gauss_legendre(n):
    xi, w = np.polynomial.legendre.leggauss(int(n))
    return xi, w


def comb(n, k):
    return math.comb(n, k)
