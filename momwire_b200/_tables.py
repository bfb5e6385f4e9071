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
    the edge's anchors, h = |edge| / n (``bspline.py:1027-1050``)."""
    sl, sr, tg, hh, rr, ed, pe = [], [], [], [], [], [], []
    e_first, e_n, e_h, e_r = [], [], [], []
    w_first, w_n, w_arc = [], [], []
    off = 0
    e_idx = 0
    for w, (pl, counts) in enumerate(zip(wires, npe)):
        start = off
        hw = []
        for e in range(pl.shape[0] - 1):
            p0, p1 = pl[e], pl[e + 1]
            vec = p1 - p0
            L = float(np.linalg.norm(vec))
            if L < 1e-15:
                raise ValueError(f"wire {w} edge {e} has zero length")
            n = int(counts[e])
            t = np.linspace(0.0, 1.0, n + 1)
            pts = (1 - t[:, None]) * p0[None, :] + t[:, None] * p1[None, :]
            sl.append(pts[:-1])
            sr.append(pts[1:])
            tg.append(np.tile(vec / L, (n, 1)))
            h = L / n
            hh.append(np.full(n, h))
            hw.append(np.full(n, h))
            rr.append(np.full(n, float(radius_per_wire[w])))
            ed.append(np.full(n, e_idx, dtype=np.int32))
            pe.append(np.arange(n, dtype=np.int32))
            e_first.append(off)
            e_n.append(n)
            e_h.append(h)
            e_r.append(float(radius_per_wire[w]))
            e_idx += 1
            off += n
        w_first.append(start)
        w_n.append(off - start)
        w_arc.append(np.concatenate([[0.0], np.cumsum(np.concatenate(hw))]))
    return Geometry(
        seg_l=np.ascontiguousarray(np.vstack(sl)),
        seg_r=np.ascontiguousarray(np.vstack(sr)),
        tangents=np.ascontiguousarray(np.vstack(tg)),
        h=np.concatenate(hh),
        radius=np.concatenate(rr),
        edge=np.concatenate(ed),
        pos_in_edge=np.concatenate(pe),
        edge_first=np.asarray(e_first, dtype=np.int32),
        edge_n=np.asarray(e_n, dtype=np.int32),
        edge_h=np.asarray(e_h, dtype=np.float64),
        edge_radius=np.asarray(e_r, dtype=np.float64),
        wire_first=np.asarray(w_first, dtype=np.int64),
        wire_n=np.asarray(w_n, dtype=np.int64),
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


@dataclass
class Basis:
    degree: int
    supp: np.ndarray  # (n_b, d+1) int32, -1 = padded wing
    polys: np.ndarray  # (n_b, d+1, d+1)
    kcl_A: "scipy.sparse.csr_matrix"  # (n_c, n_b) KCL rows, entries +-1
    knots: list  # per wire
    kept: list  # per wire: list of (j_local, kind, junction, end, m_global)

    @property
    def n(self) -> int:
        return int(self.supp.shape[0])


def build_basis(geom: Geometry, degree, start_status, end_status, n_junctions, grounded) -> Basis:
    """Clamped knot vector per wire; keep interior bases plus the value-1
    end basis at junction / ground ends; per-wing monomial coefficients in
    local arc length from values at d+1 uniform points (the reference's
    design-matrix + Vandermonde step, ``bspline.py:1318-1414``)."""
    d = int(degree)
    supp_all, poly_all, knots_all, kept_all = [], [], [], []
    jdirs = {j: [] for j in range(n_junctions)}
    m = 0
    for w in range(len(geom.wire_first)):
        arc = geom.wire_arc[w]
        n_w = int(geom.wire_n[w])
        first = int(geom.wire_first[w])
        knots = np.concatenate([np.zeros(d), arc, np.full(d, arc[-1])])
        knots_all.append(knots)
        n_b = n_w + d
        kept = []
        if start_status[w] == "ground":
            kept.append((0, "gnd", None, "start"))
        elif start_status[w] != "free":
            kept.append((0, "dir", start_status[w], "start"))
        kept.extend((j, "int", None, None) for j in range(1, n_b - 1))
        if end_status[w] == "ground":
            kept.append((n_b - 1, "gnd", None, "end"))
        elif end_status[w] != "free":
            kept.append((n_b - 1, "dir", end_status[w], "end"))
        # per-segment coefficients of the active bases, shape (n_w, d+1, d+1):
        # [segment, active basis c (= j - s), power p]
        hs = np.diff(arc)
        unit = np.linspace(0.0, 1.0, d + 1)
        us = hs[:, None] * unit[None, :]  # (n_w, d+1) local sample points
        spans = np.arange(n_w) + d
        vals = _span_values(knots, d, np.repeat(spans, d + 1), (arc[:-1, None] + us).ravel())
        vals = vals.reshape(n_w, d + 1, d + 1)  # [s, sample, c]
        V = us[:, :, None] ** np.arange(d + 1)[None, None, :]  # [s, sample, p]
        coef = np.linalg.solve(V, vals)  # [s, p, c]
        coef = np.transpose(coef, (0, 2, 1))  # [s, c, p]
        js = np.array([k[0] for k in kept], dtype=np.int64)
        nk = len(kept)
        supp = np.full((nk, d + 1), -1, dtype=np.int32)
        poly = np.zeros((nk, d + 1, d + 1))
        lo = np.maximum(0, js - d)  # first wing of basis j
        hi = np.minimum(n_w, js + 1)  # one past its last wing
        for a in range(d + 1):
            s = lo + a
            ok = s < hi
            supp[ok, a] = first + s[ok]
            poly[ok, a, :] = coef[s[ok], (js - s)[ok], :]
        for idx, (j, kind, junc, end) in enumerate(kept):
            if kind == "dir":
                jdirs[junc].append((m + idx, 1.0 if end == "start" else -1.0))
        kept_all.append([(j, kind, junc, end, m + idx) for idx, (j, kind, junc, end) in enumerate(kept)])
        supp_all.append(supp)
        poly_all.append(poly)
        m += nk
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
        supp=np.ascontiguousarray(np.concatenate(supp_all, axis=0)),
        polys=np.ascontiguousarray(np.concatenate(poly_all, axis=0)),
        kcl_A=kcl,
        knots=knots_all,
        kept=kept_all,
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
    wings touch at most ``max_seg`` distinct segments."""
    n_b = supp.shape[0]
    firsts, nbs, segs = [], [], []
    m = 0
    while m < n_b:
        cur = set()
        cnt = 0
        while m + cnt < n_b and cnt < max_basis:
            s = {int(x) for x in supp[m + cnt] if x >= 0}
            if len(cur | s) > max_seg:
                break
            cur |= s
            cnt += 1
        if cnt == 0:
            raise ValueError("a single basis touches more segments than a tile holds")
        firsts.append(m)
        nbs.append(cnt)
        segs.append(sorted(cur))
        m += cnt
    T = len(firsts)
    used = max(len(s) for s in segs) if segs else 1
    seg_arr = np.full((T, used), -1, dtype=np.int32)
    loc = np.full(supp.shape, -1, dtype=np.int32)
    for t, (f, c, s) in enumerate(zip(firsts, nbs, segs)):
        seg_arr[t, : len(s)] = s
        pos = {v: i for i, v in enumerate(s)}
        for mm in range(f, f + c):
            for a in range(supp.shape[1]):
                if supp[mm, a] >= 0:
                    loc[mm, a] = pos[int(supp[mm, a])]
    return Tiles(
        first=np.asarray(firsts, dtype=np.int32),
        nb=np.asarray(nbs, dtype=np.int32),
        ns=np.asarray([len(s) for s in segs], dtype=np.int32),
        seg=seg_arr,
        loc=loc,
        max_basis=int(max(nbs)),
        max_seg=int(used),
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
