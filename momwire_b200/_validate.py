"""Constructor checks of the port and connection keywords, table-driven.

``feeds=``, ``junctions=``, ``junction_ports=`` and ``node_gaps=`` are each
checked entry by entry against an ordered table of rules.  A rule looks at
one entry (and at what the earlier entries left in the shared state) and
returns the refusal text when the entry breaks it, ``None`` otherwise; the
first broken rule raises ``ValueError`` with that text.  The texts and the
order in which problems are reported are the reference's interface
(``bspline.py:727-960``); ``tests/golden/refusals.json`` pins them.  Entries
that pass are returned in the normalised form the solver stores:

* feeds: ``(wire, arclength or None, complex voltage)``;
* junctions: lists of ``(wire, "start"|"end")``;
* junction ports: ``(junction, complex voltage)`` (a bare index means 0 V);
* node gaps: ``(wire, "start"|"end", complex voltage)``.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

_ENDS = ("start", "end")


def _check(rules, entry):
    for rule in rules:
        text = rule(entry)
        if text is not None:
            raise ValueError(text)


# ------------------------------------------------------------------ feeds
def _feed_shape(e):
    if len(e.raw) != 3:
        return f"feeds[{e.i}]: expected (wire_index, arclength, voltage), got {e.raw!r}"
    e.wire, e.arc, e.volt = e.raw
    return None


def _feed_wire(e):
    if not 0 <= e.wire < e.n_wires:
        return f"feeds[{e.i}]: wire_index {e.wire} out of range [0, {e.n_wires})"
    return None


FEED_RULES = (_feed_shape, _feed_wire)


def feeds(entries, n_wires, feed_wire_index, feed_arclength, other_ports):
    """Normalised feed list; ``entries is None`` means the single default
    feed (``feed_wire_index``, ``feed_arclength``, 1 V)."""
    if entries is None:
        if not 0 <= feed_wire_index < n_wires:
            raise ValueError(f"feed_wire_index {feed_wire_index} out of range")
        return [(int(feed_wire_index), feed_arclength, 1.0 + 0.0j)]
    if not len(entries) and not other_ports:
        raise ValueError("feeds must contain at least one entry")
    out = []
    for i, raw in enumerate(entries):
        e = SimpleNamespace(i=i, raw=raw, n_wires=n_wires)
        _check(FEED_RULES, e)
        out.append((int(e.wire), None if e.arc is None else float(e.arc), complex(e.volt)))
    return out


# -------------------------------------------------------------- junctions
def _member_wire(e):
    if not 0 <= e.wire < e.n_wires:
        return f"junction {e.j}: wire_idx {e.wire} out of range [0, {e.n_wires})"
    return None


def _member_end(e):
    if e.end not in _ENDS:
        return f"junction {e.j}: end must be 'start' or 'end', got {e.end!r}"
    return None


MEMBER_RULES = (_member_wire, _member_end)


def junctions(groups, n_wires):
    """Normalised junction groups (a one-member group is legal: a lone-end
    attachment)."""
    out = []
    for j, group in enumerate(groups or ()):
        if len(group) < 1:
            raise ValueError(f"junction {j}: need >= 1 wire-end")
        members = []
        for w, end in group:
            _check(MEMBER_RULES, SimpleNamespace(j=j, wire=w, end=end, n_wires=n_wires))
            members.append((int(w), end))
        out.append(members)
    return out


def junction_anchor_check(groups, polylines, n_per_edge):
    """Members of a junction must meet at one point: each within
    max(1e-5 m, 1e-3 x the shortest terminal segment of the group) of the
    first member's end (``_wire_spec.py:62``).  A wrong wire index in a
    group would otherwise weld distant ends into a well-posed wrong model."""
    for j, group in enumerate(groups):
        pts, seg_len = [], []
        for w, end in group:
            pl, counts = np.asarray(polylines[w], dtype=float), n_per_edge[w]
            tip, nxt, cnt = (pl[0], pl[1], counts[0]) if end == "start" else (pl[-1], pl[-2], counts[-1])
            pts.append(tip)
            seg_len.append(float(np.linalg.norm(nxt - tip)) / max(int(cnt), 1))
        tol = max(1e-5, 1e-3 * min(seg_len))
        gaps = np.linalg.norm(np.asarray(pts[1:]) - pts[0], axis=1) if len(pts) > 1 else np.zeros(0)
        far = np.flatnonzero(gaps > tol)
        if far.size:
            k = int(far[0]) + 1
            (w0, e0), (w, e) = group[0], group[k]
            raise ValueError(
                f"junction {j}: members do not coincide - wire {w} {e} at {tuple(pts[k])} is "
                f"{float(gaps[k - 1]):.6g} m from wire {w0} {e0} at {tuple(pts[0])} (tolerance {tol:.3g} m, 1e-3 "
                "of the shortest terminal segment; a junction group must name ONE point - momwire#522)"
            )


# --------------------------------------------------------- junction ports
def _jport_range(e):
    if not 0 <= e.junction < e.n_junctions:
        return f"junction_ports: junction index {e.junction} out of range [0, {e.n_junctions})"
    return None


def _jport_once(e):
    if e.junction in e.state.ported:
        return f"junction_ports: junction {e.junction} listed twice"
    return None


JUNCTION_PORT_RULES = (_jport_range, _jport_once)


def junction_ports(entries, n_junctions):
    state = SimpleNamespace(ported=set())
    out = []
    for raw in entries or ():
        bare = isinstance(raw, (int, np.integer))
        e = SimpleNamespace(junction=int(raw if bare else raw[0]), volt=0j if bare else complex(raw[1]),
                            n_junctions=n_junctions, state=state)
        _check(JUNCTION_PORT_RULES, e)
        state.ported.add(e.junction)
        out.append((e.junction, e.volt))
    return out


# -------------------------------------------------------------- node gaps
def _gap_shape(e):
    if len(e.raw) != 3:
        return f"node_gaps[{e.i}]: expected (wire_index, 'start'|'end', voltage), got {e.raw!r}"
    e.wire, e.end, e.volt = e.raw
    return None


def _gap_wire(e):
    if not 0 <= e.wire < e.n_wires:
        return f"node_gaps[{e.i}]: wire_index {e.wire} out of range [0, {e.n_wires})"
    return None


def _gap_end(e):
    if e.end not in _ENDS:
        return f"node_gaps[{e.i}]: end must be 'start' or 'end', got {e.end!r}"
    return None


def _gap_at_junction(e):
    e.member = (int(e.wire), e.end)
    e.junction = e.state.owner.get(e.member)
    if e.junction is None:
        return (f"node_gaps[{e.i}]: wire {e.wire} {e.end!r} is not a member of any junction group — a series "
                "node gap lives at a junction; for a feed inside a wire use feeds=")
    return None


def _gap_through_path(e):
    if e.state.sizes[e.junction] < 2:
        return (f"node_gaps[{e.i}]: junction {e.junction} has a single member — there is no through-current "
                "path to be in series with (a lone-end attachment is junction_ports=)")
    return None


def _gap_member_once(e):
    if e.member in e.state.members:
        return f"node_gaps[{e.i}]: wire {e.wire} {e.end!r} listed twice"
    return None


def _gap_junction_once(e):
    if e.junction in e.state.gapped:
        return f"node_gaps[{e.i}]: junction {e.junction} already carries a node gap — one series gap per junction"
    return None


def _gap_not_shunt_port(e):
    if e.junction in e.state.ported:
        return (f"node_gaps[{e.i}]: junction {e.junction} is also a junction port — the shunt (#172) and series "
                "(#305) ports of one node cannot be driven together yet")
    return None


NODE_GAP_RULES = (_gap_shape, _gap_wire, _gap_end, _gap_at_junction, _gap_through_path, _gap_member_once,
                  _gap_junction_once, _gap_not_shunt_port)


def node_gaps(entries, n_wires, groups, ports):
    """Series gaps at junction nodes, each naming the member wire-end it is
    in series with."""
    state = SimpleNamespace(owner={m: j for j, g in enumerate(groups) for m in g},
                            sizes=[len(g) for g in groups], ported={j for j, _v in ports},
                            members=set(), gapped=set())
    out = []
    for i, raw in enumerate(entries or ()):
        e = SimpleNamespace(i=i, raw=raw, n_wires=n_wires, state=state)
        _check(NODE_GAP_RULES, e)
        state.members.add(e.member)
        state.gapped.add(e.junction)
        out.append((int(e.wire), e.end, complex(e.volt)))
    return out


# --------------------------------------------------------- scalar settings
_VARIANTS = ("raw", "stable", "tikhonov", "auto")

# (broken when, exception, text) over the keyword dict, in report order
SETTING_RULES = (
    (lambda k: k["degree"] < 1, ValueError, lambda k: f"degree must be >= 1, got {k['degree']}"),
    (lambda k: k["degree"] > 2, NotImplementedError,
     lambda k: "degree > 2 needs scripts/derive_bspline_static_moments.py to be re-run with a larger MAX_D"),
    (lambda k: not k["wires"], ValueError, lambda k: "wires must be non-empty"),
    (lambda k: k["use_singular_enrichment"] and k["enrichment_loading"], NotImplementedError,
     lambda k: k["enrichment_loading_refusal"]),
    (lambda k: k["enrichment_variant"] not in _VARIANTS, ValueError,
     lambda k: f"enrichment_variant must be one of 'raw', 'stable', 'tikhonov', 'auto', got "
               f"{k['enrichment_variant']!r}"),
    (lambda k: k["precision"] not in ("fp64", "mixed"), ValueError,
     lambda k: f"precision must be 'fp64' or 'mixed', got {k['precision']!r}"),
    (lambda k: k["sommerfeld_method"] not in ("grid", "surrogate"), ValueError,
     lambda k: f"sommerfeld_method must be 'grid' or 'surrogate', got {k['sommerfeld_method']!r}"),
    (lambda k: k["ground_eps"] is not None and k["ground_z"] is None, ValueError,
     lambda k: "ground_eps requires ground_z to be set"),
    (lambda k: k["ground_phi_mode"] not in k["phi_modes"], ValueError,
     lambda k: f"ground_phi_mode must be one of {tuple(k['phi_modes'])}, got {k['ground_phi_mode']!r}"),
    (lambda k: k["ground_model"] not in ("refl-coef", "sommerfeld"), ValueError,
     lambda k: f"ground_model must be 'refl-coef' or 'sommerfeld', got {k['ground_model']!r}"),
    (lambda k: k["ground_model"] == "sommerfeld" and k["ground_eps"] is None, ValueError,
     lambda k: "ground_model='sommerfeld' requires ground_eps"),
    (lambda k: int(k["swept_mem_mb"]) < 1, ValueError,
     lambda k: f"swept_mem_mb must be >= 1, got {k['swept_mem_mb']}"),
    (lambda k: k["feed_model"] not in ("point", "segment"), ValueError,
     lambda k: f"feed_model must be 'point' or 'segment', got {k['feed_model']!r}"),
    (lambda k: k["feed_model"] == "segment" and k["feed_smoothing_factor"] is not None, ValueError,
     lambda k: "feed_model='segment' and feed_smoothing_factor are mutually exclusive — both replace the point "
               "drive with a spread one"),
    (lambda k: bool(k["extended_kernel"]) and k["use_singular_enrichment"], NotImplementedError,
     lambda k: k["enrichment_ek_refusal"]),
)


def settings(keywords):
    """Raise for the first scalar keyword the rule table refuses."""
    for broken, exc, text in SETTING_RULES:
        if broken(keywords):
            raise exc(text(keywords))


# ---------------------------------------------------------------- wires
def polylines(wires):
    """Each wire as an (M, 3) float array with M >= 2."""
    out = [np.asarray(w, dtype=float) for w in wires]
    bad = [i for i, pl in enumerate(out) if pl.ndim != 2 or pl.shape[0] < 2 or pl.shape[1] != 3]
    if bad:
        raise ValueError(f"wire {bad[0]}: polyline must be (M, 3) with M >= 2")
    return out


def radii(wire_radius, n_wires):
    """One positive finite radius per wire (a scalar is broadcast)."""
    r = np.asarray(wire_radius, dtype=float)
    if r.ndim == 0:
        r = np.full(n_wires, float(r))
    elif r.shape != (n_wires,):
        raise ValueError(f"wire_radius: expected a scalar or a length-{n_wires} sequence (one entry per wire), "
                         f"got shape {r.shape}")
    if not (np.isfinite(r).all() and (r > 0.0).all()):
        raise ValueError(f"wire_radius entries must be positive and finite, got {r}")
    return r


def edge_counts(lines, per_wire, nsegs):
    """Segments per straight edge, per wire: None means ``nsegs`` on every
    edge, a scalar applies to every edge of its wire."""
    n_wires = len(lines)
    per_wire = [None] * n_wires if per_wire is None else per_wire
    if len(per_wire) != n_wires:
        raise ValueError(f"n_per_edge_per_wire length {len(per_wire)} != n_wires {n_wires}")
    out = []
    for i, (pl, spec) in enumerate(zip(lines, per_wire)):
        n_edges = pl.shape[0] - 1
        spec = nsegs if spec is None else spec
        counts = [int(spec)] * n_edges if np.isscalar(spec) else list(spec)
        if len(counts) != n_edges:
            raise ValueError(f"wire {i}: n_per_edge length {len(counts)} != n_edges {n_edges}")
        out.append(counts)
    return out
