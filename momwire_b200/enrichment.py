"""Host side of singular basis enrichment (``use_singular_enrichment``).

At every junction of at least ``enrichment_min_k`` wire ends the reference
adds one basis per wire end, on the segment beside the junction, shaped
u log u (u the distance from the junction over the segment length) --
minus, for the "stable" variant, its L2 projection onto the degree-d
polynomials that vanish at both ends of the segment -- and solves the
augmented system [[Z, Z_pe], [Z_ep, Z_ee]] (``bspline.py:3048-3693``,
``4121-4179``).  The blocks are filled on the device (``mw_enrich_blocks``);
this module holds the specs, the shape's polynomial, the Sommerfeld
remainder reaction of the enrichment bases, the "auto" variant's tap
ratios and the shapes' contribution to currents between knots.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _tables as T


@dataclass(frozen=True)
class Spec:
    """One enrichment basis (``bspline.py:3048-3076``)."""

    junction: int
    wire: int
    end: str  # "start" or "end"
    seg: int  # global segment beside the junction
    origin: int  # 0: the junction is the segment's left end, 1: its right end


def specs(junctions, geom: T.Geometry, min_k: int, active=None) -> list[Spec]:
    """Enrichment bases in junction order, member order within a junction;
    ``active`` (junction indices) restricts them for the "auto" variant."""
    keep = None if active is None else set(active)
    out = []
    for j, members in enumerate(junctions):
        if len(members) < min_k or (keep is not None and j not in keep):
            continue
        for w, end in members:
            first = int(geom.wire_first[w])
            last = first + int(geom.wire_n[w]) - 1
            out.append(Spec(j, int(w), end, first if end == "start" else last, 0 if end == "start" else 1))
    return out


def bubble_projection(d: int) -> np.ndarray:
    """Monomial coefficients c of the L2-orthogonal projection of t log t
    onto {p in P_d : p(0) = p(1) = 0} on [0, 1] (``bspline.py:233-300``).

    That subspace is spanned by b_i = t^(i+1) (1 - t), i = 0 .. d-2, so the
    projection solves the (d-1)-square normal equations with
    <b_i, b_j> = 1/(s+3) - 2/(s+4) + 1/(s+5) (s = i + j) and
    <t log t, b_i> = 1/(i+4)^2 - 1/(i+3)^2 (from int t^n log t = -1/(n+1)^2).
    Empty below degree 2: the stable shape is then the raw one."""
    c = np.zeros(d + 1)
    if d < 2:
        return c
    idx = np.arange(d - 1)
    s = idx[:, None] + idx[None, :]
    gram = 1.0 / (s + 3) - 2.0 / (s + 4) + 1.0 / (s + 5)
    rhs = 1.0 / (idx + 4.0) ** 2 - 1.0 / (idx + 3.0) ** 2
    a = np.linalg.solve(gram, rhs)
    c[1:d] += a
    c[2:d + 1] -= a
    return c


def shape_polynomial(variant: str, d: int) -> np.ndarray:
    """P of the shape u log u - P(u): zero for "raw", "tikhonov" and "auto"
    (the latter two change the solve, not the shape)."""
    return bubble_projection(d) if variant == "stable" else np.zeros(d + 1)


def gauss01(n: int):
    """Gauss-Legendre nodes and weights on [0, 1] (the reference's
    ``leggauss`` mapped as t = (x + 1) / 2, w / 2)."""
    x, w = np.polynomial.legendre.leggauss(int(n))
    return 0.5 * (x + 1.0), 0.5 * w


def shape_values(sp: list[Spec], geom: T.Geometry, t: np.ndarray, poly: np.ndarray):
    """(points (E, q, 3), shape value (E, q)) of each basis at nodes t."""
    pts = np.empty((len(sp), t.size, 3))
    val = np.empty((len(sp), t.size))
    for i, s in enumerate(sp):
        u = t if s.origin == 0 else 1.0 - t
        val[i] = u * np.log(np.maximum(u, 1e-300)) - np.polynomial.polynomial.polyval(u, poly)
        pts[i] = geom.seg_l[s.seg] + t[:, None] * (geom.seg_r[s.seg] - geom.seg_l[s.seg])
    return pts, val


def tap_ratios(junctions, knot_currents, min_k: int):
    """min |I| / max |I| over the wire ends meeting at each junction, read at
    the junction-side knot of each wire (``bspline.py:3078-3112``); None
    below min_k ends."""
    out = []
    for members in junctions:
        if len(members) < min_k:
            out.append(None)
            continue
        mags = [abs(knot_currents[w][0 if end == "start" else -1]) for w, end in members]
        top = max(mags)
        out.append(0.0 if top == 0.0 else min(mags) / top)
    return out


def add_between_knots(currents, coeffs, sp: list[Spec], geom: T.Geometry, s_eval, poly, n_poly):
    """Add each enrichment shape's current at the evaluation arcs inside its
    segment (it vanishes at both bounding knots) (``bspline.py:4649-4683``)."""
    for i, s in enumerate(sp):
        w = s.wire
        local = s.seg - int(geom.wire_first[w])
        arc = geom.wire_arc[w]
        lo, hi = arc[local], arc[local + 1]
        se = s_eval[w]
        mask = (se >= lo) & (se <= hi)
        if not np.any(mask):
            continue
        u = ((se[mask] - lo) if s.origin == 0 else (hi - se[mask])) / geom.h[s.seg]
        phi = np.zeros_like(u)
        pos = u > 0.0
        phi[pos] = u[pos] * np.log(u[pos])
        if np.any(poly != 0.0):
            phi = phi - np.polynomial.polynomial.polyval(u, poly)
        currents[w][mask] = currents[w][mask] + coeffs[n_poly + i] * phi
    return currents
