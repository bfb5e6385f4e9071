"""CPU oracle for momwire's B-spline Galerkin dense-solve path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this module, and only as the
checker.  The product package ``momwire_b200`` never imports it.

This is a plain numpy/scipy restatement of the reference algorithm, written
for clarity rather than speed.  Each function cites the reference routine it
restates (paths are relative to the momwire source tree, ``src/momwire/``).
It is pinned against the reference's own known-answer tests (the pins in
``tests/test_oracle_pins.py``) and against golden vectors produced by running
the reference itself (``tests/golden/make_golden.py``).

One deliberate difference from the reference: the same-edge *static* moments
(the reference evaluates sympy-generated closed forms,
``_bspline_static_moments.py`` / ``_bspline_ek_moments.py``) are evaluated
here by reducing the double integral to a one-dimensional convolution with a
piecewise-polynomial weight and integrating that with geometrically graded
Gauss-Legendre panels.  Both are evaluations of the same integral; the tests
bound the difference.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg

# bspline.py:151-152 (the solver's own vacuum constants; c = 1/sqrt(eps*mu)).
EPS0 = 8.8541878188e-12
MU0 = 1.25663706127e-6
C0 = 1.0 / math.sqrt(EPS0 * MU0)
INV4PI = 1.0 / (4.0 * math.pi)


def gl01(n):
    """Gauss-Legendre nodes/weights on [0, 1] (``_quadrature.py:27`` + the
    ``t01 = (xi+1)/2`` mapping of ``_bspline_kernels.py:658-660``)."""
    xi, w = np.polynomial.legendre.leggauss(int(n))
    return 0.5 * (xi + 1.0), 0.5 * w


# ---------------------------------------------------------------------------
# Problem specification (the subset of BSplineSolver.__init__ this path uses)
# ---------------------------------------------------------------------------


@dataclass
class Spec:
    """Normalised solver inputs; mirrors ``BSplineSolver.__init__``
    (``bspline.py:511-982``) for the served subset."""

    wires: list
    npe: list  # per wire: list of per-edge segment counts
    degree: int = 2
    feeds: list = field(default_factory=list)  # (wire, arc|None, V)
    feed_model: str = "point"
    junctions: list = field(default_factory=list)
    junction_ports: list = field(default_factory=list)  # (junction, V)
    node_gaps: list = field(default_factory=list)  # (wire, end, V)
    n_qp_pair: int = 4
    n_qp_source: int = 16
    extended_kernel: bool = False
    wavelength: float = 22.0
    radius: np.ndarray = None  # per wire
    ground_z: float | None = None
    ground_eps: object = None
    ground_phi_mode: str = "normal"
    ground_model: str = "refl-coef"
    n_qp_sommerfeld: int = 3
    wire_conductivity: np.ndarray | None = None  # per wire, NaN = off
    insulation_radius: np.ndarray | None = None
    insulation_eps_r: np.ndarray | None = None

    @property
    def k(self):
        freq = C0 / self.wavelength
        return 2 * math.pi * freq / C0

    @property
    def omega(self):
        return 2 * math.pi * (C0 / self.wavelength)


def make_spec(
    *,
    wires,
    nsegs=101,
    n_per_edge_per_wire=None,
    degree=2,
    feeds=None,
    feed_wire_index=0,
    feed_arclength=None,
    feed_model="point",
    junctions=None,
    junction_ports=None,
    node_gaps=None,
    n_qp_pair=4,
    n_qp_source=16,
    extended_kernel=False,
    wavelength=22,
    wire_radius=0.0005,
    ground_z=None,
    ground_eps=None,
    ground_phi_mode="normal",
    ground_model="refl-coef",
    n_qp_sommerfeld=3,
    wire_conductivity=None,
    insulation_radius=None,
    insulation_eps_r=None,
):
    """Build a :class:`Spec` from BSplineSolver-style kwargs
    (``bspline.py:402-637``: per-edge counts, feeds, junction ports)."""
    wires = [np.asarray(w, dtype=float) for w in wires]
    n_w = len(wires)
    if n_per_edge_per_wire is None:
        n_per_edge_per_wire = [None] * n_w
    npe = []
    for pl, e in zip(wires, n_per_edge_per_wire):
        n_e = pl.shape[0] - 1
        if e is None:
            e = nsegs
        if np.isscalar(e):
            e = [int(e)] * n_e
        npe.append([int(x) for x in e])
    if feeds is None:
        feeds = [(feed_wire_index, feed_arclength, 1.0)]
    feeds = [(int(w), None if a is None else float(a), complex(v)) for w, a, v in feeds]
    jn = [[(int(w), e) for w, e in g] for g in (junctions or [])]
    jp = []
    for p in junction_ports or []:
        if isinstance(p, (int, np.integer)):
            jp.append((int(p), 0j))
        else:
            jp.append((int(p[0]), complex(p[1])))
    ng = [(int(w), e, complex(v)) for w, e, v in (node_gaps or [])]
    r = np.asarray(wire_radius, dtype=float)
    if r.ndim == 0:
        r = np.full(n_w, float(r))
    return Spec(
        wires=wires,
        npe=npe,
        degree=int(degree),
        feeds=feeds,
        feed_model=feed_model,
        junctions=jn,
        junction_ports=jp,
        node_gaps=ng,
        n_qp_pair=int(n_qp_pair),
        n_qp_source=int(n_qp_source),
        extended_kernel=bool(extended_kernel),
        wavelength=float(wavelength),
        radius=r,
        ground_z=ground_z,
        ground_eps=ground_eps,
        ground_phi_mode=ground_phi_mode,
        ground_model=ground_model,
        n_qp_sommerfeld=int(n_qp_sommerfeld),
        wire_conductivity=_per_wire(wire_conductivity, n_w),
        insulation_radius=_per_wire(insulation_radius, n_w),
        insulation_eps_r=_per_wire(insulation_eps_r, n_w),
    )


def _per_wire(v, n_w):
    if v is None:
        return None
    a = np.asarray(v, dtype=float)
    return np.full(n_w, float(a)) if a.ndim == 0 else a


# ---------------------------------------------------------------------------
# Geometry  (bspline.py:988-1093)
# ---------------------------------------------------------------------------


def build_geometry(spec):
    """Uniform segmentation of each polyline edge (``bspline.py:1027-1050``)."""
    seg_l, seg_r, tan, h, radius = [], [], [], [], []
    wires_info = []
    edges = []  # (first global segment, n segments, h, radius, wire)
    off = 0
    for w, (pl, npe) in enumerate(zip(spec.wires, spec.npe)):
        w_first = off
        h_w = []
        for e in range(pl.shape[0] - 1):
            p0, p1 = pl[e], pl[e + 1]
            L = float(np.linalg.norm(p1 - p0))
            if L < 1e-15:
                raise ValueError(f"wire {w} edge {e} has zero length")
            n = npe[e]
            t = np.linspace(0.0, 1.0, n + 1)
            pts = (1 - t[:, None]) * p0[None, :] + t[:, None] * p1[None, :]
            seg_l.append(pts[:-1])
            seg_r.append(pts[1:])
            tan.append(np.tile((p1 - p0) / L, (n, 1)))
            h.append(np.full(n, L / n))
            h_w.append(np.full(n, L / n))
            radius.append(np.full(n, spec.radius[w]))
            edges.append((off, n, L / n, float(spec.radius[w]), w))
            off += n
        h_w = np.concatenate(h_w)
        wires_info.append(
            {"first": w_first, "n": off - w_first, "arc": np.concatenate([[0.0], np.cumsum(h_w)])}
        )
    return {
        "seg_l": np.vstack(seg_l),
        "seg_r": np.vstack(seg_r),
        "tangents": np.vstack(tan),
        "h": np.concatenate(h),
        "radius": np.concatenate(radius),
        "wires": wires_info,
        "edges": edges,
        "n": off,
    }


def _touch_tol(pl):
    """``_ground_spec.py:127-153``: 1e-6 of the polyline length."""
    length = float(np.sum(np.linalg.norm(np.diff(pl, axis=0), axis=1)))
    return 1e-6 * max(length, 1e-30)


def endpoint_status(spec):
    """``bspline.py:1108-1150``: free / ground / junction index per wire end."""
    n_w = len(spec.wires)
    st = ["free"] * n_w
    en = ["free"] * n_w
    for j, g in enumerate(spec.junctions):
        for w, e in g:
            if e == "start":
                st[w] = j
            else:
                en[w] = j
    if spec.ground_z is not None:
        gz = spec.ground_z
        for w, pl in enumerate(spec.wires):
            tol = _touch_tol(pl)
            at = np.abs(pl[:, 2] - gz) <= tol
            if st[w] == "free" and at[0]:
                st[w] = "ground"
            if en[w] == "free" and at[-1]:
                en[w] = "ground"
    return st, en


def grounded_junctions(spec):
    """``bspline.py:1152-1169``."""
    if spec.ground_z is None:
        return set()
    out = set()
    for j, g in enumerate(spec.junctions):
        w, e = g[0]
        pl = spec.wires[w]
        pt = pl[0] if e == "start" else pl[-1]
        if abs(pt[2] - spec.ground_z) <= _touch_tol(pl):
            out.add(j)
    return out


def span_basis_values(knots, d, span, x):
    """Values of the d+1 B-splines that are nonzero on knot span ``span``
    at points ``x`` (the span's own polynomial pieces, evaluated even at the
    span's right end).  Classic triangular Cox-de Boor recursion."""
    x = np.atleast_1d(np.asarray(x, dtype=float))
    N = np.zeros((x.size, d + 1))
    N[:, 0] = 1.0
    left = np.zeros((x.size, d + 1))
    right = np.zeros((x.size, d + 1))
    for j in range(1, d + 1):
        left[:, j] = x - knots[span + 1 - j]
        right[:, j] = knots[span + j] - x
        saved = np.zeros(x.size)
        for r in range(j):
            tmp = N[:, r] / (right[:, r + 1] + left[:, j - r])
            N[:, r] = saved + right[:, r + 1] * tmp
            saved = left[:, j - r] * tmp
        N[:, j] = saved
    return N  # column c <-> basis (span - d + c)


def eval_bspline_basis(knots, d, x):
    """All basis values of a clamped spline at points x: (len(x), n_basis).
    Right-open spans; the last knot maps into the last non-empty span."""
    x = np.atleast_1d(np.asarray(x, dtype=float))
    n_b = len(knots) - d - 1
    out = np.zeros((x.size, n_b))
    for i, xv in enumerate(x):
        span = int(np.searchsorted(knots, xv, side="right")) - 1
        span = min(max(span, d), n_b - 1)
        vals = span_basis_values(knots, d, span, xv)[0]
        out[i, span - d : span + 1] = vals
    return out


@dataclass
class Basis:
    supp_seg: np.ndarray  # (n_b, d+1) int64, padded wings -> 0
    polys: np.ndarray  # (n_b, d+1, d+1), padded wings -> 0
    kcl_A: np.ndarray  # (n_c, n_b)
    knots: list
    kept: list  # per wire: list of (j_local, kind, junction, end, m_global)


def build_basis(spec, geom):
    """Per-(basis, wing) monomial coefficients in local arc length u,
    support map, KCL rows (``bspline.py:1216-1414``)."""
    d = spec.degree
    st, en = endpoint_status(spec)
    supp, polys, knots_all, kept_all = [], [], [], []
    jdirs = {j: [] for j in range(len(spec.junctions))}
    m = 0
    for w, info in enumerate(geom["wires"]):
        arc = info["arc"]
        n_w = info["n"]
        knots = np.concatenate([np.zeros(d), arc, np.full(d, arc[-1])])
        knots_all.append(knots)
        n_b = n_w + d
        kept = []
        if st[w] == "ground":
            kept.append((0, "gnd", None, "start"))
        elif st[w] != "free":
            kept.append((0, "dir", st[w], "start"))
        for j in range(1, n_b - 1):
            kept.append((j, "int", None, None))
        if en[w] == "ground":
            kept.append((n_b - 1, "gnd", None, "end"))
        elif en[w] != "free":
            kept.append((n_b - 1, "dir", en[w], "end"))
        # per-segment monomial coefficients of the d+1 active bases
        coef = np.zeros((n_w, d + 1, d + 1))  # [s, c(active idx), p]
        for s in range(n_w):
            span = s + d
            hs = arc[s + 1] - arc[s]
            us = np.linspace(0.0, hs, d + 1)
            vals = span_basis_values(knots, d, span, arc[s] + us)  # (d+1 pts, d+1 bases)
            V = np.vander(us, d + 1, increasing=True)
            coef[s] = np.linalg.solve(V, vals).T
        wire_kept = []
        for j, kind, junc, end in kept:
            lo, hi = max(0, j - d), min(n_w, j + 1)
            sm = np.zeros(d + 1, dtype=np.int64)
            pm = np.zeros((d + 1, d + 1))
            for a, s in enumerate(range(lo, hi)):
                sm[a] = info["first"] + s
                pm[a] = coef[s, j - s]
            supp.append(sm)
            polys.append(pm)
            if kind == "dir":
                jdirs[junc].append((m, 1.0 if end == "start" else -1.0))
            wire_kept.append((j, kind, junc, end, m))
            m += 1
        kept_all.append(wire_kept)
    grounded = grounded_junctions(spec)
    rows = [j for j in range(len(spec.junctions)) if j not in grounded]
    kcl = np.zeros((len(rows), m))
    for r, j in enumerate(rows):
        for mg, sg in jdirs[j]:
            kcl[r, mg] = sg
    return Basis(
        supp_seg=np.array(supp, dtype=np.int64).reshape(m, d + 1),
        polys=np.array(polys).reshape(m, d + 1, d + 1),
        kcl_A=kcl,
        knots=knots_all,
        kept=kept_all,
    )


# ---------------------------------------------------------------------------
# Extended-kernel eligibility  (_bspline_kernels.py:198-321)
# ---------------------------------------------------------------------------


def ek_factor(R, a, k):
    """NEC Eq 89 coaxial factor 1 + T1*C2 - T2*C1 (``_bspline_kernels.py:198``)."""
    kr = k * R
    c1 = 1.0 + 1j * kr
    c2 = 3.0 * c1 - kr * kr
    t1 = 0.25 * a**4 / R**4
    t2 = 0.5 * a**2 / R**2
    return 1.0 + t1 * c2 - t2 * c1


def ek_reg_extra(R, a, k):
    """fac - fac_static (``_bspline_kernels.py:225``)."""
    kr = k * R
    t1 = 0.25 * a**4 / R**4
    t2 = 0.5 * a**2 / R**2
    return t1 * (3j * kr - kr * kr) - t2 * (1j * kr)


def ek_axis_groups(seg_l, seg_r, tangents, seg_a, tol=1e-6):
    """Coaxial-and-equal-radius labels (``_bspline_kernels.py:249-321``):
    a segment joins the first earlier group whose representative is
    (anti)parallel, of equal radius and on the same axis."""
    centers = 0.5 * (seg_l + seg_r)
    labels = np.empty(len(seg_a), dtype=np.int64)
    reps = []  # (center, tangent, radius)
    for i in range(len(seg_a)):
        hit = -1
        for g, (c, t, a) in enumerate(reps):
            if abs(float(t @ tangents[i])) < 1.0 - tol:
                continue
            if abs(seg_a[i] / a - 1.0) > tol:
                continue
            dv = centers[i] - c
            perp = dv - (dv @ tangents[i]) * tangents[i]
            if np.linalg.norm(perp) <= tol * a:
                hit = g
                break
        if hit < 0:
            hit = len(reps)
            reps.append((centers[i], tangents[i], seg_a[i]))
        labels[i] = hit
    return labels


def mirror_pts(p, gz):
    """``_ground_mirror.py:37``."""
    q = p.copy()
    q[..., 2] = 2 * gz - q[..., 2]
    return q


def ek_labels(spec, geom, mirror):
    """``bspline.py:2040-2088``: joint scan over real + mirrored segments."""
    sl, sr, t, a = geom["seg_l"], geom["seg_r"], geom["tangents"], geom["radius"]
    if not mirror:
        lab = ek_axis_groups(sl, sr, t, a)
        return lab, lab
    n = len(a)
    tm = t * np.array([1.0, 1.0, -1.0])
    joint = ek_axis_groups(
        np.vstack([sl, mirror_pts(sl, spec.ground_z)]),
        np.vstack([sr, mirror_pts(sr, spec.ground_z)]),
        np.vstack([t, tm]),
        np.concatenate([a, a]),
    )
    return joint[:n], joint[n:]


# ---------------------------------------------------------------------------
# Moments
# ---------------------------------------------------------------------------


def offedge_moments(sl_i, sr_i, sl_j, sr_j, a_row, k, d, nq, groups=None, rows_per_chunk=64):
    """Full-kernel GL moments on every segment pair
    (``_bspline_kernels.py:599-747``; C++ ``_accelerators.cpp:370-542``).

    J[p, P, i, j] = sum_{q,r} w_q u_q^p w_r u_r^P exp(-jkR)/(4 pi R),
    R^2 = |x_iq - x_jr|^2 + a_i^2 (observer-row radius); on pairs with equal
    EK labels the Eq 89 factor multiplies the kernel.
    """
    t, w = gl01(nq)
    n_i, n_j = sl_i.shape[0], sl_j.shape[0]
    Li = np.linalg.norm(sr_i - sl_i, axis=1)
    Lj = np.linalg.norm(sr_j - sl_j, axis=1)
    pi = (1 - t[None, :, None]) * sl_i[:, None, :] + t[None, :, None] * sr_i[:, None, :]
    pj = (1 - t[None, :, None]) * sl_j[:, None, :] + t[None, :, None] * sr_j[:, None, :]
    wu_i = np.stack([(w * Li[:, None]) * (t * Li[:, None]) ** p for p in range(d + 1)])
    wu_j = np.stack([(w * Lj[:, None]) * (t * Lj[:, None]) ** p for p in range(d + 1)])
    a_row = np.broadcast_to(np.asarray(a_row, dtype=float), (n_i,))
    J = np.empty((d + 1, d + 1, n_i, n_j), dtype=np.complex128)
    for i0 in range(0, n_i, rows_per_chunk):
        i1 = min(n_i, i0 + rows_per_chunk)
        diff = pi[i0:i1, :, None, None, :] - pj[None, None, :, :, :]
        a2 = (a_row[i0:i1] ** 2)[:, None, None, None]
        R = np.sqrt((diff * diff).sum(-1) + a2)
        G = np.exp(-1j * k * R) / (4 * np.pi * R)
        if groups is not None:
            gi, gj = groups
            mask = gi[i0:i1, None] == gj[None, :]
            fac = ek_factor(R, a_row[i0:i1][:, None, None, None], k)
            G = np.where(mask[:, None, :, None], G * fac, G)
        J[:, :, i0:i1, :] = np.einsum("piq,iqjr,Pjr->pPij", wu_i[:, i0:i1], G, wu_j, optimize=True)
    return J


def _graded_panels(lo, hi, peak, a, ratio=2.0):
    """Split [lo, hi] into panels graded geometrically (scale ``a``) away
    from ``peak`` (the kernel's near-singular point)."""
    pts = {lo, hi}
    if lo < peak < hi:
        pts.add(peak)
    out = sorted(pts)
    panels = []
    for x0, x1 in zip(out[:-1], out[1:]):
        dist = min(abs(x0 - peak), abs(x1 - peak))
        if dist >= (x1 - x0):
            panels.append((x0, x1))
            continue
        # grade toward whichever end is nearer the peak
        near_left = abs(x0 - peak) <= abs(x1 - peak)
        L = x1 - x0
        cuts = [0.0]
        s = max(a, 1e-300)
        while s < L:
            cuts.append(s)
            s *= ratio
        cuts.append(L)
        for c0, c1 in zip(cuts[:-1], cuts[1:]):
            if near_left:
                panels.append((x0 + c0, x0 + c1))
            else:
                panels.append((x1 - c1, x1 - c0))
    return panels


def _conv_weight(p, q, h, tt):
    """W_pq(t) = integral of u^p (u - t)^q du over the overlap of [0,h] and
    [t, h+t], for t in [-h, h] (vectorised over tt).  Expanded so every term
    is non-negative: for t >= 0 substitute v = u - t (u^p = (v+t)^p), for
    t < 0 expand (u + |t|)^q."""
    tt = np.asarray(tt, dtype=float)
    acc = np.zeros_like(tt)
    pos = tt >= 0
    tp, tn = tt[pos], -tt[~pos]
    for r in range(p + 1):
        e = q + r + 1
        acc[pos] += math.comb(p, r) * tp ** (p - r) * (h - tp) ** e / e
    for r in range(q + 1):
        e = p + r + 1
        acc[~pos] += math.comb(q, r) * tn ** (q - r) * (h - tn) ** e / e
    return acc


def same_edge_static_table(h, a, n, d, ek=False, n_gl=20):
    """Static same-edge moments as a Toeplitz table over delta = j - i
    (restates ``_bspline_kernels.py:333-422`` + the generated closed forms).

    S_pq(delta) = (1/4pi) * int_0^h int_0^h u^p v^q K(u - v - delta*h) dv du,
    K(x) = 1/sqrt(x^2 + a^2)  [+ EK: -a^2/(2R^3) + 3a^4/(4R^5)].
    Reduced to int_{-h}^{h} W_pq(t) K(t - delta*h) dt with graded GL panels.
    Returns (2n-1, d+1, d+1), index delta + n - 1.
    """
    xg, wg = np.polynomial.legendre.leggauss(n_gl)
    out = np.zeros((2 * n - 1, d + 1, d + 1))
    for di, delta in enumerate(range(-(n - 1), n)):
        c = delta * h
        nodes, weights = [], []
        for lo, hi in ((-h, 0.0), (0.0, h)):
            for x0, x1 in _graded_panels(lo, hi, c, a):
                half = 0.5 * (x1 - x0)
                nodes.append(0.5 * (x0 + x1) + half * xg)
                weights.append(half * wg)
        tt = np.concatenate(nodes)
        ww = np.concatenate(weights)
        x = tt - c
        R = np.sqrt(x * x + a * a)
        K = 1.0 / R
        if ek:
            K = K + (a * a / (4.0 * R**5)) * (3.0 * a * a - 2.0 * R * R)
        for p in range(d + 1):
            for q in range(d + 1):
                out[di, p, q] = INV4PI * np.sum(ww * _conv_weight(p, q, h, tt) * K)
    return out


def same_edge_reg_table(h, a, n, k, d, nq, ek=False):
    """Smooth same-edge part (exp(-jkR)-1)/(4 pi R) by q x q GL per pair,
    Toeplitz in delta (``_bspline_kernels.py:425-581``; C++ ``:165-327``)."""
    t, w = gl01(nq)
    u = t * h
    wu = np.stack([w * h * u**p for p in range(d + 1)])  # (d+1, nq)
    out = np.zeros((2 * n - 1, d + 1, d + 1), dtype=np.complex128)
    for di, delta in enumerate(range(-(n - 1), n)):
        x = u[:, None] - u[None, :] - delta * h
        R = np.sqrt(x * x + a * a)
        if ek:
            G = ((np.exp(-1j * k * R) - 1.0) * ek_factor(R, a, k) + ek_reg_extra(R, a, k)) / (4 * np.pi * R)
        else:
            G = (np.exp(-1j * k * R) - 1.0) / (4 * np.pi * R)
        out[di] = np.einsum("pq,qr,Pr->pP", wu, G, wu)
    return out


def fill_J(spec, geom, k):
    """All-pairs moment tensor with same-edge blocks overwritten by static +
    reg (``bspline.py:2222-2283``)."""
    d = spec.degree
    groups = ek_labels(spec, geom, False) if spec.extended_kernel else None
    J = offedge_moments(geom["seg_l"], geom["seg_r"], geom["seg_l"], geom["seg_r"],
                        geom["radius"], k, d, spec.n_qp_pair, groups)
    for first, n, h, a, _w in geom["edges"]:
        st = same_edge_static_table(h, a, n, d, ek=spec.extended_kernel)
        rg = same_edge_reg_table(h, a, n, k, d, spec.n_qp_pair, ek=spec.extended_kernel)
        tab = st + rg
        idx = np.arange(n)[None, :] - np.arange(n)[:, None] + (n - 1)
        blk = tab[idx]  # (n, n, d+1, d+1)
        J[:, :, first : first + n, first : first + n] = np.transpose(blk, (2, 3, 0, 1))
    return J


def fill_J_image(spec, geom, k):
    """Moments against mirrored sources (``bspline.py:1428-1465``)."""
    gz = spec.ground_z
    groups = ek_labels(spec, geom, True) if spec.extended_kernel else None
    return offedge_moments(geom["seg_l"], geom["seg_r"], mirror_pts(geom["seg_l"], gz),
                           mirror_pts(geom["seg_r"], gz), geom["radius"], k, spec.degree,
                           spec.n_qp_pair, groups)


# ---------------------------------------------------------------------------
# Galerkin assembly  (bspline.py:2289-2348, 1684-1734)
# ---------------------------------------------------------------------------


def assemble(J, basis, omega, wA, wPhi=None):
    """Z = j w mu sum_ab wA * (C J C) + (1/(j w eps)) sum_ab wPhi * (C' J C').

    ``wA`` is the per-segment-pair A-term table (tangent dot for free space),
    ``wPhi`` the per-pair charge-term weight (None = 1)."""
    supp, polys = basis.supp_seg, basis.polys
    nb, nw, npoly = polys.shape
    d = npoly - 1
    ZA = np.zeros((nb, nb), dtype=np.complex128)
    ZP = np.zeros((nb, nb), dtype=np.complex128)
    pv = np.arange(1, d + 1, dtype=float)
    for a in range(nw):
        sm = supp[:, a]
        for b in range(nw):
            sn = supp[:, b]
            Jb = J[:, :, sm[:, None], sn[None, :]]
            ZA += wA[sm[:, None], sn[None, :]] * np.einsum("mp,pPmn,nP->mn", polys[:, a, :], Jb, polys[:, b, :])
            dm = polys[:, a, 1:] * pv[None, :]
            dn = polys[:, b, 1:] * pv[None, :]
            inner = np.einsum("mp,pPmn,nP->mn", dm, Jb[:d, :d], dn)
            ZP += inner if wPhi is None else wPhi[sm[:, None], sn[None, :]] * inner
    return 1j * omega * MU0 * ZA + ZP / (1j * omega * EPS0)


# ---------------------------------------------------------------------------
# Grounds  (_ground_spec.py:90-126, _ground_refl.py, _potential_ground.py)
# ---------------------------------------------------------------------------


def eps_tilde(ground_eps, omega):
    """``_ground_refl.py:46-60``."""
    if isinstance(ground_eps, (tuple, list)):
        er, sig = ground_eps
        return complex(float(er), -float(sig) / (omega * EPS0))
    return complex(ground_eps)


def image_weights(spec, geom, omega):
    """(w_A, w_Phi) tables for the image block of each ground model
    (``_potential_ground.py:711-810``)."""
    t = geom["tangents"]
    tm = t * np.array([1.0, 1.0, -1.0])
    td_img = t @ tm.T
    if spec.ground_eps is None:
        return td_img.astype(np.complex128), None
    et = eps_tilde(spec.ground_eps, omega)
    if spec.ground_model == "sommerfeld":
        c2 = (et - 1.0) / (et + 1.0)
        return c2 * td_img, np.full(td_img.shape, c2, dtype=np.complex128)
    c = 0.5 * (geom["seg_l"] + geom["seg_r"])
    dx = c[:, 0][:, None] - c[:, 0][None, :]
    dy = c[:, 1][:, None] - c[:, 1][None, :]
    dz = c[:, 2][:, None] + c[:, 2][None, :] - 2.0 * spec.ground_z
    hyp = np.hypot(dx, dy)
    rmag = np.maximum(np.sqrt(dx * dx + dy * dy + dz * dz), 1e-30)
    cos_th = dz / rmag
    safe = hyp > 1e-30
    inv = 1.0 / np.where(safe, hyp, 1.0)
    px = np.where(safe, -dy * inv, 1.0)
    py = np.where(safe, dx * inv, 0.0)
    tm_p = t[:, 0][:, None] * px + t[:, 1][:, None] * py
    tn_p = t[:, 0][None, :] * px + t[:, 1][None, :] * py
    P = tm_p * tn_p
    sin2 = 1.0 - cos_th * cos_th
    root = np.sqrt(et - sin2 + 0j)
    rho_v = (et * cos_th - root) / (et * cos_th + root)
    rho_h = (cos_th - root) / (cos_th + root)
    wA = rho_v * (td_img - P) - rho_h * P
    mode = spec.ground_phi_mode
    if mode == "rho_v":
        wP = rho_v
    elif mode == "image":
        wP = np.full(wA.shape, (et - 1.0) / (et + 1.0))
    elif mode == "normal":
        r = np.sqrt(et)
        wP = np.full(wA.shape, (r - 1.0) / (r + 1.0))
    elif mode == "blend":
        wP = 0.5 * (rho_v + (et - 1.0) / (et + 1.0))
    else:
        raise ValueError(mode)
    return wA, wP


def sommerfeld_grid(spec, geom, master_values=None):
    """The remainder grid a Sommerfeld solve interpolates
    (``bspline.py:1781-1789``, ``1861-1862``)."""
    from oracle import sommerfeld_oracle as so

    r1_max = so.max_image_distance(geom["seg_l"], geom["seg_r"], spec.ground_z)
    et = eps_tilde(spec.ground_eps, spec.omega)
    return so.get_grid(et, spec.k, r1_max, spec.omega, MU0, master_values=master_values)


def compute_Z(spec, geom=None, basis=None, somm_master_values=None):
    """Free-space (+ image) Z for one k (``bspline.py:3702-3776``).  For the
    Sommerfeld ground the C2 image and the remainder block Q are summed
    before the one subtraction (``_potential_ground.py:524-527``);
    ``somm_master_values`` supplies the grid master's tables."""
    geom = geom or build_geometry(spec)
    basis = basis or build_basis(spec, geom)
    k, om = spec.k, spec.omega
    t = geom["tangents"]
    Z = assemble(fill_J(spec, geom, k), basis, om, (t @ t.T).astype(np.complex128))
    if spec.ground_z is not None:
        wA, wP = image_weights(spec, geom, om)
        img = assemble(fill_J_image(spec, geom, k), basis, om, wA, wP)
        if spec.ground_eps is not None and spec.ground_model == "sommerfeld":
            from oracle import sommerfeld_oracle as so

            grid = sommerfeld_grid(spec, geom, somm_master_values)
            img = img + so.remainder_Q(geom, basis.supp_seg, basis.polys, spec.degree, spec.n_qp_sommerfeld,
                                       spec.ground_z, k, grid)
        Z -= img
    if loading_active(spec):
        Z = Z + loading_matrix(spec, geom, basis, om)
    return Z


# ---------------------------------------------------------------------------
# Distributed series wire loading  (_wire_loading.py; bspline.py:2667-2760)
# ---------------------------------------------------------------------------


def loading_active(spec):
    return spec.wire_conductivity is not None or spec.insulation_radius is not None


def internal_impedance(omega, a, sigma):
    """Round solid conductor, Z' = k_c / (2 pi a sigma) I0(k_c a) / I1(k_c a),
    k_c = sqrt(j omega mu0 sigma) (``_wire_loading.py``
    ``wire_internal_impedance``).  Unscaled Bessels: valid while |k_c a|
    stays well below the overflow of I_n (a / skin depth < ~300)."""
    from scipy.special import iv

    kc = np.sqrt(1j * omega * MU0 * sigma)
    return kc / (2 * math.pi * a * sigma) * iv(0, kc * a) / iv(1, kc * a)


def z_per_wire(spec, omega):
    """Z'_w(omega) per wire (``_wire_loading.py`` ``series_impedance_per_wire``)."""
    n_w = len(spec.wires)
    out = np.zeros(n_w, dtype=np.complex128)
    for w in range(n_w):
        a = spec.radius[w]
        if spec.wire_conductivity is not None and np.isfinite(spec.wire_conductivity[w]):
            out[w] += internal_impedance(omega, a, spec.wire_conductivity[w])
        if spec.insulation_radius is not None and np.isfinite(spec.insulation_radius[w]):
            b, er = spec.insulation_radius[w], spec.insulation_eps_r[w]
            out[w] += 1j * omega * MU0 / (2 * math.pi) * (1 - 1 / er) * math.log(b / a)
    return out


def loading_gram(geom, basis):
    """Dense S with S[m, n] = integral of Phi_m Phi_n over the segments both
    bases cover, per wire: (n_wires, n_b, n_b).  Each shared segment is
    integrated with (d+1)-point Gauss-Legendre, exact for the degree-2d
    product (``bspline.py:2667-2731`` forms the same moment in closed form)."""
    supp, polys = basis.supp_seg, basis.polys
    n_b, n_wing, n_p = polys.shape
    wire_of_seg = np.concatenate([np.full(w["n"], i) for i, w in enumerate(geom["wires"])])
    x, wq = gl01(n_p)
    by_seg = {}
    for m in range(n_b):
        for a in range(n_wing):
            if np.any(polys[m, a] != 0.0):
                by_seg.setdefault(int(supp[m, a]), []).append((m, a))
    S = np.zeros((len(geom["wires"]), n_b, n_b))
    for sgm, ents in by_seg.items():
        h = geom["h"][sgm]
        u = h * x
        vals = [np.polyval(polys[m, a][::-1], u) for m, a in ents]
        for i, (m, _a) in enumerate(ents):
            for j, (n, _b) in enumerate(ents):
                S[wire_of_seg[sgm], m, n] += h * np.sum(wq * vals[i] * vals[j])
    return S


def loading_matrix(spec, geom, basis, omega):
    """sum_w Z'_w(omega) S_w (``bspline.py:2732-2753``)."""
    S = loading_gram(geom, basis)
    return np.einsum("w,wmn->mn", z_per_wire(spec, omega), S)


# ---------------------------------------------------------------------------
# Ports and solve  (bspline.py:2806-3050, 3778-3867, 4053-4179)
# ---------------------------------------------------------------------------


def port_columns(spec, geom, basis):
    """B = [gap feeds | junction-port KCL rows | node-gap indicators] and
    the remaining KCL constraint rows (``bspline.py:3841-3867``)."""
    d = spec.degree
    nb = basis.supp_seg.shape[0]
    cols = []
    for w, arc_req, _v in spec.feeds:
        arc = geom["wires"][w]["arc"]
        s_f = arc_req if arc_req is not None else arc[-1] / 2.0
        knots = basis.knots[w]
        if spec.feed_model == "point":
            vals = eval_bspline_basis(knots, d, [s_f])[0]
        else:  # "segment": (1/h) * integral over the cell holding s_f
            s = int(np.searchsorted(arc, s_f, side="right")) - 1
            s = max(0, min(s, len(arc) - 2))
            lo, hi = arc[s], arc[s + 1]
            xg, wg = np.polynomial.legendre.leggauss(spec.n_qp_source)
            tt = 0.5 * (hi + lo) + 0.5 * (hi - lo) * xg
            vals = (eval_bspline_basis(knots, d, tt).T @ (0.5 * (hi - lo) * wg)) / (hi - lo)
        v = np.zeros(nb, dtype=np.complex128)
        for j, _kind, _jn, _end, mg in basis.kept[w]:
            v[mg] = vals[j]
        cols.append(v)
    B = np.array(cols, dtype=np.complex128).reshape(len(cols), nb).T
    # junction ports (bspline.py:1171-1214)
    grounded = grounded_junctions(spec)
    row_of, r = {}, 0
    for j in range(len(spec.junctions)):
        if j not in grounded:
            row_of[j] = r
            r += 1
    port_rows = [row_of[j] for j, _v in spec.junction_ports]
    keep = [i for i in range(basis.kcl_A.shape[0]) if i not in set(port_rows)]
    kcl_con = basis.kcl_A[keep, :]
    port_A = basis.kcl_A[port_rows, :]
    # node gaps (bspline.py:3784-3818)
    e2j = {}
    for j, g in enumerate(spec.junctions):
        for mem in g:
            e2j[mem] = j
    gap = np.zeros((nb, len(spec.node_gaps)))
    for p, (w, end, _v) in enumerate(spec.node_gaps):
        j = e2j[(w, end)]
        for _jl, kind, jn, en, mg in basis.kept[w]:
            if kind == "dir" and jn == j and en == end:
                gap[mg, p] = 1.0 if end == "start" else -1.0
    return np.hstack([B, port_A.T.astype(np.complex128), gap.astype(np.complex128)]), kcl_con


def solve_ports(Z, B, kcl_con):
    """``_solve_with_kcl_ports`` (``bspline.py:2971-2989``)."""
    if kcl_con.shape[0] == 0:
        return scipy.linalg.solve(Z, B)
    n_p = B.shape[1]
    sol = scipy.linalg.solve(Z, np.hstack([B, kcl_con.T.astype(np.complex128)]))
    W, X = sol[:, :n_p], sol[:, n_p:]
    Lam = scipy.linalg.solve(kcl_con @ X, kcl_con @ W)
    return W - X @ Lam


def port_solution(spec, somm_master_values=None):
    """``compute_port_solution`` (``bspline.py:4053-4179``): returns
    (Y, coeffs, Z, geom, basis)."""
    geom = build_geometry(spec)
    basis = build_basis(spec, geom)
    Z = compute_Z(spec, geom, basis, somm_master_values)
    B, kcl = port_columns(spec, geom, basis)
    X = solve_ports(Z, B, kcl)
    return B.T @ X, X, Z, geom, basis


def currents_at_knots(spec, geom, basis, coeffs):
    """``bspline.py:4586-4685`` (no enrichment): per-wire current at knots."""
    d = spec.degree
    out = []
    for w, info in enumerate(geom["wires"]):
        knots = basis.knots[w]
        s = np.clip(info["arc"], knots[0], knots[-1])
        c = np.zeros(len(knots) - d - 1, dtype=np.complex128)
        for j, _k, _jn, _e, mg in basis.kept[w]:
            c[j] = coeffs[mg]
        out.append(eval_bspline_basis(knots, d, s) @ c)
    return out
