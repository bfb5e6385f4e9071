"""Distributed series wire loading: conductor loss and insulation.

A non-PEC wire carries a series impedance per unit length Z'_w(omega):

* the internal impedance of a round solid conductor of radius a and
  conductivity sigma, Z'_int = k_c / (2 pi a sigma) * I0(k_c a) / I1(k_c a)
  with k_c = sqrt(j omega mu0 sigma), exact from DC to strong skin effect
  (``_wire_loading.py`` ``wire_internal_impedance``).  The Bessel ratio is
  taken from exponentially scaled Bessels, whose common factor cancels;
* the quasi-static jacket inductance of a dielectric insulation (inner
  radius a, outer b, relative permittivity eps_r),
  L' = mu0 / (2 pi) * (1 - 1/eps_r) * ln(b/a)
  (``_wire_loading.py`` ``insulation_inductance``).

The Galerkin B-spline testing turns it into Z += sum_w Z'_w(omega) S_w with
S the same-wire basis-overlap Gram S[m, n] = integral Phi_m Phi_n dl, a
closed-form polynomial moment per shared segment
(``bspline.py:2667-2760``: ``_loading_gram``, ``_apply_loading``).  The Gram
is k-independent: it is built once per structure on the host (a few entries
per basis), coalesced, uploaded, and every fill adds it scaled by that
frequency's per-wire Z' with one small device kernel (``mw_add_loading``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.special import ive

MU0 = 1.25663706127e-6


def wire_internal_impedance(omega, radius, sigma):
    """Per-unit-length internal impedance of a round solid conductor [Ohm/m]
    (``_wire_loading.py`` ``wire_internal_impedance``)."""
    omega = np.asarray(omega, dtype=float)
    if radius <= 0.0:
        raise ValueError(f"wire radius must be > 0, got {radius}")
    if sigma <= 0.0:
        raise ValueError(f"conductivity must be > 0 S/m, got {sigma}")
    kc = np.sqrt(1j * omega * MU0 * sigma)
    x = kc * radius
    return kc / (2.0 * np.pi * radius * sigma) * (ive(0, x) / ive(1, x))


def insulation_inductance(radius, ins_radius, eps_r):
    """Series inductance per unit length of a dielectric jacket [H/m]
    (``_wire_loading.py`` ``insulation_inductance``)."""
    if ins_radius <= radius:
        raise ValueError(f"insulation_radius ({ins_radius}) must exceed the conductor radius ({radius})")
    if eps_r < 1.0:
        raise ValueError(f"insulation_eps_r must be >= 1, got {eps_r}")
    return MU0 / (2.0 * np.pi) * (1.0 - 1.0 / eps_r) * np.log(ins_radius / radius)


def normalize_per_wire(value, n_wires, name):
    """None | scalar | one entry per wire -> None | (n_wires,) float array;
    NaN entries switch a wire off (``_wire_loading.py`` ``normalize_per_wire``)."""
    if value is None:
        return None
    arr = np.asarray(value, dtype=float)
    if arr.ndim == 0:
        arr = np.full(n_wires, float(arr))
    if arr.shape != (n_wires,):
        raise ValueError(
            f"{name}: expected a scalar or a length-{n_wires} sequence (one entry per wire), got shape {arr.shape}"
        )
    return arr


@dataclass
class WireLoading:
    """Normalised loading configuration: each field None (off) or a
    (n_wires,) array with NaN switching a wire off."""

    radius: np.ndarray
    conductivity: np.ndarray | None
    insulation_radius: np.ndarray | None
    insulation_eps_r: np.ndarray | None

    def z_wire(self, omega):
        """Z'_w(omega) [Ohm/m]: (n_wires,) for a scalar omega, (n_wires, n_k)
        for an array (``_wire_loading.py`` ``series_impedance_per_wire``)."""
        omega = np.asarray(omega, dtype=float)
        n_w = self.radius.shape[0]
        out = np.zeros((n_w,) + omega.shape, dtype=np.complex128)
        for w in range(n_w):
            if self.conductivity is not None and np.isfinite(self.conductivity[w]):
                out[w] += wire_internal_impedance(omega, self.radius[w], self.conductivity[w])
            if self.insulation_radius is not None and np.isfinite(self.insulation_radius[w]):
                ell = insulation_inductance(self.radius[w], self.insulation_radius[w], self.insulation_eps_r[w])
                out[w] += 1j * omega * ell
        return out


def configure(n_wires, radius_per_wire, wire_conductivity, insulation_radius, insulation_eps_r):
    """Validate the three loading keywords in the reference's order and with
    its messages (``_wire_loading.py`` ``configure_loading``).  Returns a
    ``WireLoading`` or None when no loading is configured."""
    cond = normalize_per_wire(wire_conductivity, n_wires, "wire_conductivity")
    ins_r = normalize_per_wire(insulation_radius, n_wires, "insulation_radius")
    ins_e = normalize_per_wire(insulation_eps_r, n_wires, "insulation_eps_r")
    if (ins_r is None) != (ins_e is None):
        raise ValueError("insulation_radius and insulation_eps_r must be given together")
    radius = np.asarray(radius_per_wire, dtype=float)
    if ins_r is not None:
        finite = np.isfinite(ins_r)
        if not np.array_equal(finite, np.isfinite(ins_e)):
            raise ValueError(
                "insulation_radius and insulation_eps_r must be finite on the same wires "
                "(NaN switches a wire off in both)"
            )
        for w in np.nonzero(finite)[0]:
            insulation_inductance(radius[w], ins_r[w], ins_e[w])
    if cond is not None:
        for w in np.nonzero(np.isfinite(cond))[0]:
            if cond[w] <= 0.0:
                raise ValueError(f"wire_conductivity[{w}] must be > 0 S/m, got {cond[w]}")
    if cond is None and ins_r is None:
        return None
    return WireLoading(radius=radius, conductivity=cond, insulation_radius=ins_r, insulation_eps_r=ins_e)


@dataclass
class LoadingGram:
    """Same-wire basis-overlap Gram.  ``rows, cols, vals, wire`` are the
    per-shared-segment triplets (duplicates add up, as the reference's COO);
    ``u_*`` the coalesced unique (row, col) entries the device adds."""

    rows: np.ndarray
    cols: np.ndarray
    vals: np.ndarray
    wire: np.ndarray
    u_rows: np.ndarray
    u_cols: np.ndarray
    u_vals: np.ndarray
    u_wire: np.ndarray


def loading_gram(geom, basis) -> LoadingGram:
    """S[m, n] = sum over shared segments of sum_pq C[m,a,p] C[n,b,q]
    h^(p+q+1)/(p+q+1) (``bspline.py:2667-2731``), all segments at once:
    the (basis, wing) pairs are grouped by segment (at most d+1 per
    segment) and each segment's block is C H C^T."""
    supp, polys = basis.supp, basis.polys
    n_b, n_w, n_p = polys.shape
    live = (supp >= 0) & np.any(polys != 0.0, axis=2)
    mm, aa = np.nonzero(live)
    seg = supp[mm, aa].astype(np.int64)
    order = np.lexsort((aa, mm, seg))
    mm, aa, seg = mm[order], aa[order], seg[order]
    if seg.size == 0:
        z = np.zeros(0, dtype=np.int64)
        return LoadingGram(z, z, np.zeros(0), z, z, z, np.zeros(0), z)
    used, start, count = np.unique(seg, return_index=True, return_counts=True)
    K = int(count.max())
    slot = np.arange(seg.size) - np.repeat(start, count)
    S = used.size
    C = np.zeros((S, K, n_p))
    M_idx = np.full((S, K), -1, dtype=np.int64)
    srow = np.repeat(np.arange(S), count)
    C[srow, slot] = polys[mm, aa]
    M_idx[srow, slot] = mm
    pq = np.arange(n_p)
    pq_sum = (pq[:, None] + pq[None, :] + 1).astype(float)
    H = geom.h[used][:, None, None] ** pq_sum[None] / pq_sum[None]
    M = np.einsum("sip,spq,sjq->sij", C, H, C)
    ok = (M_idx[:, :, None] >= 0) & (M_idx[:, None, :] >= 0)
    s_i, i_i, j_i = np.nonzero(ok)
    rows = M_idx[s_i, i_i]
    cols = M_idx[s_i, j_i]
    vals = M[s_i, i_i, j_i]
    wire_of_seg = np.repeat(np.arange(len(geom.wire_n)), geom.wire_n)
    wire = wire_of_seg[used[s_i]]
    key = rows * n_b + cols
    ukey, inv = np.unique(key, return_inverse=True)
    u_vals = np.bincount(inv, weights=vals, minlength=ukey.size)
    u_wire = np.zeros(ukey.size, dtype=np.int64)
    u_wire[inv] = wire
    return LoadingGram(rows=rows, cols=cols, vals=vals, wire=wire, u_rows=ukey // n_b, u_cols=ukey % n_b,
                       u_vals=u_vals, u_wire=u_wire)
