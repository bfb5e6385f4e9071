"""What holds each wire end, which junctions sit on the ground, and which
constraint rows become ports -- as index arrays.

The reference answers these three questions with per-wire loops
(``bspline.py:1108-1214``).  Here the answer is one integer table: ``ends``
has a row per wire and a column per end (0 = start, 1 = end) holding the
junction index that owns the end, ``FREE`` or ``GROUND``.  A junction takes
precedence over the ground; an end that touches the ground plane (within
``_tables.touch_tol``) and belongs to no junction is grounded.  The KCL
port split reads the junction of each constraint row that the basis
builder recorded (``Basis.kcl_junction``) instead of recounting rows.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse

from . import _tables as T

FREE = -1
GROUND = -2
_SIDE = {"start": 0, "end": 1}


def _ground_touch(polylines, ground_z):
    """Per wire: its touch tolerance, and a boolean per vertex that lies on
    the ground plane."""
    tol = np.array([T.touch_tol(pl) for pl in polylines])
    on = [np.abs(np.asarray(pl)[:, 2] - ground_z) <= t for pl, t in zip(polylines, tol)]
    return tol, on


def end_table(polylines, junctions, ground_z):
    """(n_wires, 2) int64 table of end holders; raises for a wire below the
    ground plane or an edge lying in it (checked wire by wire, a wire's dip
    before its flat edge, as the reference reports them)."""
    ends = np.full((len(polylines), 2), FREE, dtype=np.int64)
    flat = [(w, _SIDE[side], j) for j, group in enumerate(junctions) for w, side in group]
    if flat:
        w, c, j = np.array(flat, dtype=np.int64).T
        ends[w, c] = j  # a later member of the same end wins
    if ground_z is None:
        return ends
    tol, on = _ground_touch(polylines, ground_z)
    zmin = np.array([float(np.min(np.asarray(pl)[:, 2])) for pl in polylines])
    below = zmin < ground_z - tol
    flat_edge = np.array([bool(np.any(o[:-1] & o[1:])) for o in on])
    bad = np.flatnonzero(below | flat_edge)
    if bad.size:
        w = int(bad[0])
        if below[w]:
            raise ValueError(f"wire {w} dips below the ground plane (min z = {zmin[w]:.6g} < ground_z = {ground_z:g})")
        raise ValueError(f"wire {w} has an edge lying in the ground plane (both endpoints at ground_z) — "
                         "degenerate over a conducting ground")
    touch = np.array([[o[0], o[-1]] for o in on], dtype=bool).reshape(-1, 2)
    ends[(ends == FREE) & touch] = GROUND
    return ends


def end_status(ends):
    """The table as the per-end labels the basis builder takes: the
    junction index, "free" or "ground"."""
    def label(v):
        return "free" if v == FREE else ("ground" if v == GROUND else int(v))

    return [label(v) for v in ends[:, 0]], [label(v) for v in ends[:, 1]]


def grounded_junctions(polylines, junctions, ground_z):
    """Junctions whose node (the first member's end) lies on the ground
    plane; their KCL rows leave the constraint set, the ground image
    carrying the current."""
    if ground_z is None or not junctions:
        return frozenset()
    first = [g[0] for g in junctions]
    z = np.array([np.asarray(polylines[w])[0 if side == "start" else -1, 2] for w, side in first])
    tol = np.array([T.touch_tol(polylines[w]) for w, _side in first])
    return frozenset(int(j) for j in np.flatnonzero(np.abs(z - ground_z) <= tol))


def split_kcl_ports(kcl_A, kcl_junction, junction_ports, grounded):
    """(constraint rows, port rows, port voltages): the KCL rows of the
    junctions named as ports leave the constraint set and become the ports'
    drive/readout rows, in port order."""
    if not junction_ports:
        return kcl_A, scipy.sparse.csr_matrix((0, kcl_A.shape[1])), np.zeros(0, dtype=np.complex128)
    port_j = np.array([j for j, _v in junction_ports], dtype=np.int64)
    on_ground = np.flatnonzero(np.isin(port_j, np.fromiter(grounded, dtype=np.int64, count=len(grounded))))
    if on_ground.size:
        raise ValueError(
            f"junction {int(port_j[on_ground[0]])} is both grounded and a junction port — a grounded node's "
            "voltage is pinned by the ground image, so it cannot also be a driven port"
        )
    # constraint rows are in junction order, one per ungrounded junction
    rows = np.searchsorted(kcl_junction, port_j)
    keep = np.ones(kcl_A.shape[0], dtype=bool)
    keep[rows] = False
    volts = np.array([v for _j, v in junction_ports], dtype=np.complex128)
    return kcl_A[np.flatnonzero(keep), :], kcl_A[rows, :], volts
