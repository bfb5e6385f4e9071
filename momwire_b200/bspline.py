"""B200-native drop-in for momwire's ``BSplineSolver`` dense-solve path.

Same constructor keywords, the same ``feeds=`` / ``junction_ports=`` /
``node_gaps=`` port surface and the same ``PortSolution`` result as the
reference (``bspline.py:332``, ``:511``, ``:4053``).  Host code here builds
the O(N) tables (geometry, basis, ports) and drives the native library
``libmomwire_b200.so`` through its C ABI; torch tensors serve only as
device buffers.  The fill and the factorisation run on the GPU:

* ``precision="fp64"`` (default): complex128 fill and complex128 LU --
  the plain drop-in, matching the reference to ~1e-10;
* ``precision="mixed"``: complex64 factorisation on the tensor cores with
  FP64 iterative refinement against the FP64 fill.

For ``ground_model="sommerfeld"`` the remainder surfaces come from the
reference's quadrature grid (``sommerfeld_method="grid"``, the default and
the drop-in) or from the learned surrogate (``"surrogate"``), which falls
back to the grid outside its domain or when a quadrature spot check of the
structure misses ``surrogate_tol`` (relative surface error; default 1e-6,
which the shipped network does not reach, so the grid serves -- the
surrogate is an approximation at ``surrogate_tol=surrogate.APPROX_TOL``).
"""

from __future__ import annotations

import ctypes as C
from contextlib import contextmanager
from dataclasses import dataclass

import numpy as np
import scipy.sparse

from . import _lib
from . import _tables as T
from . import _topology as topo
from . import _validate as V
from . import autotune
from . import enrichment as EN
from . import loading as wl
from . import sommerfeld as somm
from . import surrogate as sur
from ._capabilities import Capabilities
from ._port_solution import PortSolution


class SolveAborted(Exception):
    """Solve was cancelled via a :class:`CancelToken`; no result was produced."""


class CancelToken:
    """One-shot cancellation flag shared with a solve (same surface as the
    reference's ``_cancel.CancelToken``).  The factorisation polls it
    between panels; the host polls it at phase seams."""

    def __init__(self):
        self._flag = np.zeros(1, dtype=np.int32)

    def cancel(self):
        self._flag[0] = 1

    @property
    def cancelled(self):
        return bool(self._flag[0])

    def raise_if_cancelled(self):
        if self._flag[0]:
            raise SolveAborted()

    @property
    def ptr(self):
        return self._flag.ctypes.data


@dataclass(frozen=True)
class _SplineBasis:
    """Opaque ``PortSolution.basis`` payload (reference ``bspline.py:288``)."""

    geom: object
    supp_seg: object
    polys: object
    wire_knots: object
    wire_basis_global: object
    n_poly: int


def _csr(rows, cols, vals, n_rows):
    """(row_ptr, col_idx, vals) int64 / int64 / complex128 of a coordinate
    list; entries of a row keep their given order."""
    rows = np.asarray(rows, dtype=np.int64)
    order = np.argsort(rows, kind="stable")
    ptr = np.zeros(n_rows + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n_rows)[:n_rows], out=ptr[1:])
    return ptr, np.ascontiguousarray(np.asarray(cols, dtype=np.int64)[order]), np.ascontiguousarray(
        np.asarray(vals, dtype=np.complex128)[order])


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("momwire_b200 needs a CUDA device (B200); none is visible")
    return torch


def _swept_y(Xt, B, A):
    """Y stack (n_k, P, P) from the swept solutions Xt (n_k, P + n_c, n),
    each X_k^T of Z_k [W | Xc] = [B | A^T]: with KCL rows the Schur step
    Lambda = (A Xc)^-1 (A W), X = W - Xc Lambda (``bspline.py:2980-2989``),
    then Y = B^T X."""
    P = B.shape[1]
    Wt = Xt[:, :P, :]
    if A.shape[0]:
        Xct = Xt[:, P:, :]
        S = np.einsum("cn,kdn->kcd", A, Xct)  # A Xc   (n_k, n_c, n_c)
        AW = np.einsum("cn,kpn->kcp", A, Wt)  # A W    (n_k, n_c, P)
        Lam = np.linalg.solve(S, AW)  # (n_k, n_c, P)
        Wt = Wt - np.einsum("kcp,kcn->kpn", Lam, Xct)
    return np.einsum("kpn,nq->kqp", Wt, B)


class _PackedTables:
    """The k-independent tables of one structure laid out in one page-locked
    host buffer (256-byte aligned pieces), ready for ONE stream-ordered
    upload.  Built on the host only (no CUDA call but the pinned
    allocation), so a helper thread can prepare the next structures while
    the GPU works: a copy per table (seventeen per structure) from pageable
    memory made each solver's set-up wait for the device, and that wait
    bounded sweeps over many structures."""

    def __init__(self, geom: T.Geometry, basis: T.Basis, tiles: T.Tiles, ek):
        torch = _torch()
        arrays, idx = [], {}

        def put(key, a, dtype):
            idx[key] = len(arrays)
            arrays.append(np.ascontiguousarray(a, dtype=dtype))

        put("seg_l", geom.seg_l, np.float64)
        put("seg_r", geom.seg_r, np.float64)
        put("tan", geom.tangents, np.float64)
        put("rad", geom.radius, np.float64)
        put("edge", geom.edge, np.int32)
        put("pos", geom.pos_in_edge, np.int32)
        if ek is not None:
            put("grp", ek[0], np.int32)
            if ek[1] is not None:
                put("grp_img", ek[1], np.int32)
        off, rows = T.edge_table_offsets(geom.edge_n)
        put("e_n", geom.edge_n, np.int32)
        put("e_off", off, np.int64)
        put("e_h", geom.edge_h, np.float64)
        put("e_r", geom.edge_radius, np.float64)
        put("supp", basis.supp, np.int32)
        put("polys", basis.polys, np.float64)
        put("t_first", tiles.first, np.int32)
        put("t_nb", tiles.nb, np.int32)
        put("t_ns", tiles.ns, np.int32)
        put("t_seg", tiles.seg, np.int32)
        put("loc", tiles.loc, np.int32)
        offs, total = [], 0
        for x in arrays:
            offs.append(total)
            total += (x.nbytes + 255) & ~255
        self.host = torch.empty(max(total, 256), dtype=torch.uint8, pin_memory=True)
        hv = self.host.numpy()
        for x, o in zip(arrays, offs):
            hv[o : o + x.nbytes] = x.view(np.uint8).reshape(-1)
        self.offset = {k: offs[i] for k, i in idx.items()}
        self.nbytes = int(sum(x.nbytes for x in arrays))
        self.rows = rows
        self.meta = (geom.n, len(geom.edge_n), int(geom.edge_n.max()), basis.degree, basis.n, len(tiles.first),
                     tiles.max_basis, tiles.max_seg)


class _DeviceTables:
    """Device copies of the k-independent tables plus their C structs: one
    stream-ordered copy of a _PackedTables buffer on the caller's current
    stream (the host buffer stays referenced until the object goes)."""

    def __init__(self, packed: _PackedTables, dev):
        devbuf = packed.host.to(dev, non_blocking=True)
        self.keep = [packed.host, devbuf]
        self.h2d_bytes = packed.nbytes
        ptr = {k: devbuf.data_ptr() + o for k, o in packed.offset.items()}
        n_seg, n_edge, max_n, degree, n_basis, n_tile, max_basis, max_seg = packed.meta
        self.seg = _lib.Segments(n_seg, ptr["seg_l"], ptr["seg_r"], ptr["tan"], ptr["rad"], ptr["edge"],
                                 ptr["pos"], ptr.get("grp"), ptr.get("grp_img"))
        self.table_rows = packed.rows
        self.edges = _lib.Edges(n_edge, ptr["e_n"], ptr["e_off"], ptr["e_h"], ptr["e_r"], packed.rows, max_n)
        self.basis = _lib.BasisT(degree, n_basis, ptr["supp"], ptr["polys"], n_tile, max_basis, max_seg,
                                 ptr["t_first"], ptr["t_nb"], ptr["t_ns"], ptr["t_seg"], ptr["loc"])


# the reference's refusals of enrichment combinations (bspline.py:308-330):
# their texts are part of the interface consumers read
_ENRICHMENT_WIRE_LOADING_REFUSAL = (
    "use_singular_enrichment + distributed wire loading together not supported yet — the enrichment bases don't "
    "carry the loading overlap term")
_ENRICHMENT_EXTENDED_KERNEL_REFUSAL = (
    "extended_kernel=True + use_singular_enrichment=True not supported yet — the enrichment DOFs bypass the moment "
    "kernels entirely (they carry their own Φ_sing quadrature), they exist only at K >= 3 junctions where NEC's own "
    "gating turns EK off, and the O(a²) tube expansion was never derived for the s^(-1/2) shapes "
    "(stevenmburns/momwire#249 follow-up C)")
_ENRICHMENT_PER_WIRE_RADIUS_REFUSAL = (
    "use_singular_enrichment + mixed per-wire radii together not supported yet — the enrichment kernels take a "
    "single radius (stevenmburns/momwire#147)")
_CONTACT_REFUSAL = "ground contact is refused under ground_model='refl-coef' (use ground_model='sommerfeld')"


class BSplineSolver:
    """Degree-d B-spline Galerkin MoM on multi-wire polylines with
    junctions, filled and factorised on a B200.

    Keyword arguments follow the reference constructor (``bspline.py:511-548``).
    Served: degree 1-2, reduced or extended thin-wire kernel, free space,
    PEC image, reflection-coefficient and Sommerfeld grounds, point/segment
    feeds, junctions, junction ports and node gaps, per-wire radii,
    distributed wire loading, singular basis enrichment at junctions.
    Additional:

    precision : "fp64" (default) or "mixed".
    device : CUDA device index or torch.device (default: current device).
    """

    # what the class serves, read by consumers before they build one
    # (``bspline.py:495-509``)
    capabilities = Capabilities(
        grounds=frozenset({"pec", "refl-coef", "sommerfeld"}),
        wire_loading=True,
        extended_kernel=True,
        junction_ports=True,
        node_gaps=True,
        per_wire_radius=True,
        singular_enrichment=True,
        refusals={
            "wire_loading+singular_enrichment": _ENRICHMENT_WIRE_LOADING_REFUSAL,
            "extended_kernel+singular_enrichment": _ENRICHMENT_EXTENDED_KERNEL_REFUSAL,
            "per_wire_radius+singular_enrichment": _ENRICHMENT_PER_WIRE_RADIUS_REFUSAL,
            "contact+refl-coef": _CONTACT_REFUSAL,
        },
    )

    eps = 8.8541878188e-12
    mu = 1.25663706127e-6

    def __init__(
        self,
        *,
        wires,
        n_per_edge_per_wire=None,
        degree=2,
        feed_wire_index=0,
        feed_arclength=None,
        feeds=None,
        feed_model="point",
        feed_smoothing_factor=None,
        junctions=None,
        junction_ports=None,
        node_gaps=None,
        n_qp_pair=4,
        n_qp_source=16,
        extended_kernel=False,
        wavelength=22,
        halfdriver_factor=0.962,
        wire_radius=0.0005,
        wire_conductivity=None,
        insulation_radius=None,
        insulation_eps_r=None,
        nsegs=101,
        ground_z=None,
        ground_eps=None,
        ground_phi_mode="normal",
        ground_model="refl-coef",
        n_qp_sommerfeld=3,
        use_singular_enrichment=False,
        n_qp_sing=32,
        enrichment_min_k=3,
        enrichment_variant="raw",
        tikhonov_lambda=1e-3,
        auto_tap_ratio_threshold=0.3,
        swept_mem_mb=256,
        cancel=None,
        precision="fp64",
        device=None,
        sommerfeld_method="grid",
        surrogate_tol=sur.DEFAULT_TOL,
    ):
        self._cancel = cancel
        V.settings(dict(degree=degree, wires=wires, use_singular_enrichment=use_singular_enrichment,
                        enrichment_loading=wire_conductivity is not None or insulation_radius is not None,
                        enrichment_loading_refusal=_ENRICHMENT_WIRE_LOADING_REFUSAL,
                        extended_kernel=extended_kernel, enrichment_ek_refusal=_ENRICHMENT_EXTENDED_KERNEL_REFUSAL,
                        enrichment_variant=enrichment_variant,
                        precision=precision, sommerfeld_method=sommerfeld_method, ground_eps=ground_eps,
                        ground_z=ground_z, ground_phi_mode=ground_phi_mode, phi_modes=_lib.PHI_MODES,
                        ground_model=ground_model, swept_mem_mb=swept_mem_mb, feed_model=feed_model,
                        feed_smoothing_factor=feed_smoothing_factor))
        # singular basis enrichment at junctions of >= enrichment_min_k ends
        self.use_singular_enrichment = bool(use_singular_enrichment)
        # the junctions the "auto" variant enriched in the last solve (None:
        # every qualifying junction), read back by currents_at_knots
        self._auto_active_junctions = None
        self.n_qp_sing = int(n_qp_sing)
        self.enrichment_min_k = int(enrichment_min_k)
        self.enrichment_variant = enrichment_variant
        self.tikhonov_lambda = float(tikhonov_lambda)
        self.auto_tap_ratio_threshold = float(auto_tap_ratio_threshold)
        self.precision = precision
        self.sommerfeld_method = sommerfeld_method
        if not float(surrogate_tol) > 0.0:
            raise ValueError(f"surrogate_tol must be > 0, got {surrogate_tol!r}")
        self.surrogate_tol = float(surrogate_tol)
        self.last_sommerfeld = None
        # mixed: stop refining once the relative error estimated to remain in
        # every port column (the last correction, times the contraction the
        # corrections show) is below this -- a third of the 1e-6 the mixed
        # path holds drive-point impedances to
        self.mixed_tol = 3e-7
        self.mixed_max_iter = 10
        self.last_refinement = None
        self.degree = int(degree)
        self.wavelength = wavelength
        self.halfdriver_factor = halfdriver_factor
        self.wire_radius = wire_radius
        self.nsegs = nsegs
        self.ground_z = ground_z
        self.ground_eps = ground_eps
        self.ground_phi_mode = ground_phi_mode
        self.ground_model = ground_model
        self.n_qp_sommerfeld = int(n_qp_sommerfeld)
        self.extended_kernel = bool(extended_kernel)
        self.swept_mem_mb = int(swept_mem_mb)
        self.feed_model = feed_model
        self.feed_smoothing_factor = feed_smoothing_factor
        self.n_qp_source = int(n_qp_source)

        # wavenumber from the solver's own c = 1 / sqrt(eps mu)
        self.c = 1 / np.sqrt(self.eps * self.mu)
        self.freq = self.c / self.wavelength
        self.omega = 2 * np.pi * self.freq
        self.k = self.omega / self.c
        self.halfdriver = self.halfdriver_factor * self.wavelength / 4

        self.wires_polylines = V.polylines(wires)
        n_w = len(self.wires_polylines)
        if self.ground_eps is not None and self.ground_model == "refl-coef":
            touching = self._contact_ends()
            if touching:
                where = ", ".join(f"wire {w} {kind}" for w, kind in touching)
                raise NotImplementedError(f"{where} lies in the ground plane: {_CONTACT_REFUSAL}")
        self._radius_per_wire = V.radii(wire_radius, n_w)
        if self.use_singular_enrichment and np.any(self._radius_per_wire != self._radius_per_wire[0]):
            raise NotImplementedError(_ENRICHMENT_PER_WIRE_RADIUS_REFUSAL)
        # distributed series loading (bspline.py:715-728): None when off
        self._loading = wl.configure(n_w, self._radius_per_wire, wire_conductivity, insulation_radius,
                                     insulation_eps_r)
        self.wire_conductivity = None if self._loading is None else self._loading.conductivity
        self.insulation_radius = None if self._loading is None else self._loading.insulation_radius
        self.insulation_eps_r = None if self._loading is None else self._loading.insulation_eps_r
        self._cached_loading = None
        self._cached_loading_dev = None
        self.n_per_edge_per_wire = V.edge_counts(self.wires_polylines, n_per_edge_per_wire, self.nsegs)

        # the port and connection keywords: entry by entry against ordered
        # rule tables (the reference's refusal texts and order)
        self.feeds = V.feeds(feeds, n_w, feed_wire_index, feed_arclength, bool(junction_ports) or bool(node_gaps))
        self.feed_wire_index = self.feeds[0][0] if self.feeds else None
        self.feed_arclength = self.feeds[0][1] if self.feeds else None
        # checked where the reference's quadrature first uses it: at the
        # solve (``_dev_tables``), with the reference's exception and text
        self.n_qp_pair = int(n_qp_pair)
        self.junctions = V.junctions(junctions, n_w)
        V.junction_anchor_check(self.junctions, self.wires_polylines, self.n_per_edge_per_wire)
        self.junction_ports = V.junction_ports(junction_ports, len(self.junctions))
        self.node_gaps = V.node_gaps(node_gaps, n_w, self.junctions, self.junction_ports)

        self._device = device
        self._cached_geometry = None
        self._cached_basis = None
        self._cached_tiles = None
        self._cached_dev = None
        self._cached_packed = None
        self._cached_ek = None
        self.last_stats = {}

    # ------------------------------------------------------------------ misc
    def _checkpoint(self):
        if self._cancel is not None:
            self._cancel.raise_if_cancelled()

    def _contact_ends(self):
        """``_ground_spec.contact_ends`` (reference ``_ground_spec.py:156``)."""
        if self.ground_z is None:
            return ()
        out = []
        for i, pl in enumerate(self.wires_polylines):
            tol = T.touch_tol(pl)
            if abs(float(pl[0, 2]) - self.ground_z) <= tol:
                out.append((i, "start"))
            if abs(float(pl[-1, 2]) - self.ground_z) <= tol:
                out.append((i, "end"))
        return tuple(sorted(out))

    def _set_k(self, kk):
        self.k = float(kk)
        self.omega = self.k * self.c
        self.wavelength = self.c / (self.omega / (2 * np.pi))

    @contextmanager
    def _k_restored(self):
        saved = (self.k, self.wavelength, self.omega)
        try:
            yield
        finally:
            self.k, self.wavelength, self.omega = saved

    # ------------------------------------------------------------ topology
    def _end_table(self):
        """(n_wires, 2) end holders: junction index, FREE or GROUND
        (``_topology.end_table``; ``bspline.py:1108-1150``)."""
        return topo.end_table(self.wires_polylines, self.junctions, self.ground_z)

    def _wire_endpoint_status(self):
        """Per-wire start and end labels (junction index, "free" or
        "ground"), the reference's ``_wire_endpoint_status`` view."""
        return topo.end_status(self._end_table())

    def _grounded_junctions(self):
        """``bspline.py:1152-1169``."""
        return topo.grounded_junctions(self.wires_polylines, self.junctions, self.ground_z)

    def _geometry(self) -> T.Geometry:
        if self._cached_geometry is None:
            self._cached_geometry = T.build_geometry(
                self.wires_polylines, self.n_per_edge_per_wire, self._radius_per_wire
            )
        return self._cached_geometry

    def _basis(self) -> T.Basis:
        if self._cached_basis is None:
            self._cached_basis = T.build_basis(
                self._geometry(), self.degree, self._end_table(), len(self.junctions), self._grounded_junctions()
            )
        return self._cached_basis

    def _ek(self):
        if not self.extended_kernel:
            return None
        if self._cached_ek is None:
            self._cached_ek = T.ek_labels(self._geometry(), self.ground_z)
        return self._cached_ek

    def _torch_device(self):
        torch = _torch()
        if self._device is None:
            return torch.device("cuda", torch.cuda.current_device())
        if isinstance(self._device, int):
            return torch.device("cuda", self._device)
        return torch.device(self._device)

    def _dev_tables(self) -> _DeviceTables:
        if self._cached_dev is None:
            # the reference refuses these at the solve: numpy's Gauss-Legendre
            # rule for a non-positive order, its native pair quadrature above
            # eight points (``_accelerators.cpp`` scratch buffers); so do the
            # device kernels here
            if self.n_qp_pair < 1:
                np.polynomial.legendre.leggauss(self.n_qp_pair)
            if self.n_qp_pair > 8:
                raise RuntimeError("n_qp > 8 not supported (scratch buffer size)")
            self._cached_dev = _DeviceTables(self._packed_tables(), self._torch_device())
        return self._cached_dev

    def _packed_tables(self) -> _PackedTables:
        """The host side of _dev_tables (geometry, basis, fill tiles, packed
        for one upload): no device work, so it can be prepared ahead."""
        if self._cached_packed is None:
            geom, basis = self._geometry(), self._basis()
            if self._cached_tiles is None:
                self._cached_tiles = T.build_tiles(basis.supp)
            self._cached_packed = _PackedTables(geom, basis, self._cached_tiles, self._ek())
        return self._cached_packed

    # --------------------------------------------------------------- ports
    def _split_kcl_ports(self, kcl_A):
        """(constraint rows, port rows, port voltages) of this solver's KCL
        rows ``kcl_A`` (``bspline.py:1171-1214``)."""
        return topo.split_kcl_ports(kcl_A, self._basis().kcl_junction, self.junction_ports,
                                    self._grounded_junctions())

    def _source_entries(self, w, s_f):
        """Nonzeros (basis indices, values) of the Galerkin drive column of
        one gap feed (``bspline.py:2806-2942``): point (v_m = Phi_m(s_f)),
        segment-wide gap, or cos^2 bump."""
        geom, basis = self._geometry(), self._basis()
        d = self.degree
        arc = geom.wire_arc[w]
        knots = basis.knots[w]
        if self.feed_smoothing_factor is None and self.feed_model == "point":
            vals = T.basis_values(knots, d, [s_f])[0]
        elif self.feed_model == "segment":
            s = int(np.searchsorted(arc, s_f, side="right")) - 1
            s = max(0, min(s, len(arc) - 2))
            lo, hi = float(arc[s]), float(arc[s + 1])
            xg, wg = T.gauss_legendre(self.n_qp_source)
            t = 0.5 * (hi + lo) + 0.5 * (hi - lo) * xg
            vals = T.basis_values(knots, d, t).T @ ((0.5 * (hi - lo) * wg) / (hi - lo))
        else:
            h = np.diff(arc)
            s = int(np.searchsorted(arc, s_f, side="right")) - 1
            s = max(0, min(s, len(h) - 1))
            width = float(self.feed_smoothing_factor) * float(h[s])
            half = width / 2.0
            lo, hi = max(0.0, s_f - half), min(float(arc[-1]), s_f + half)
            if lo >= hi:
                raise ValueError("feed_smoothing_factor too large for wire — bump doesn't fit")
            xg, wg = T.gauss_legendre(self.n_qp_source)
            t = 0.5 * (hi + lo) + 0.5 * (hi - lo) * xg
            wts = 0.5 * (hi - lo) * wg
            delta = t - s_f
            g = np.where(np.abs(delta) < half, (2.0 / width) * np.cos(np.pi * delta / width) ** 2, 0.0)
            vals = np.einsum("qj,q,q->j", T.basis_values(knots, d, t), g, wts)
        idx = np.array([mg for j, _kind, _jn, _end, mg in basis.kept[w] if vals[j] != 0.0], dtype=np.int64)
        val = np.array([vals[j] for j, _kind, _jn, _end, _mg in basis.kept[w] if vals[j] != 0.0],
                       dtype=np.complex128)
        return idx, val

    def _source_vector(self, w, s_f):
        """Dense drive column of one gap feed (see ``_source_entries``)."""
        v = np.zeros(self._basis().n, dtype=np.complex128)
        idx, val = self._source_entries(w, s_f)
        v[idx] = val
        return v

    def _node_gap_columns(self):
        """``bspline.py:3784-3818``."""
        basis = self._basis()
        cols = np.zeros((basis.n, len(self.node_gaps)))
        volts = np.zeros(len(self.node_gaps), dtype=np.complex128)
        if not self.node_gaps:
            return cols, volts
        grounded = self._grounded_junctions()
        e2j = {m: j for j, jw in enumerate(self.junctions) for m in jw}
        for p, (w, end, v) in enumerate(self.node_gaps):
            j = e2j[(w, end)]
            if j in grounded:
                raise ValueError(
                    f"node_gaps[{p}]: junction {j} is grounded — a series gap between a wire and the "
                    "ground stake is not supported"
                )
            for _jl, kind, jn, en, mg in basis.kept[w]:
                if kind == "dir" and jn == j and en == end:
                    cols[mg, p] = 1.0 if end == "start" else -1.0
            volts[p] = v
        return cols, volts

    def _port_columns(self):
        """(B, kcl_con) with ports [feeds | junction ports | node gaps]
        (``bspline.py:3841-3867``)."""
        geom, basis = self._geometry(), self._basis()
        B = np.zeros((basis.n, len(self.feeds)), dtype=np.complex128)
        for i, (w, arc_i, _v) in enumerate(self.feeds):
            s_f = arc_i if arc_i is not None else geom.wire_arc[w][-1] / 2.0
            B[:, i] = self._source_vector(w, s_f)
        kcl_con, port_A, _pv = self._split_kcl_ports(basis.kcl_A)
        gap, _gv = self._node_gap_columns()
        return np.hstack([B, port_A.T.toarray().astype(np.complex128), gap.astype(np.complex128)]), kcl_con

    def _port_entries(self):
        """(rows, cols, vals, n_p): the nonzeros of the port matrix B of
        ``_port_columns`` in coordinate form (feeds, junction-port KCL rows,
        node gaps)."""
        geom, basis = self._geometry(), self._basis()
        rs, cs, vs = [], [], []
        ws = [w for w, _a, _v in self.feeds]
        sfs = [a if a is not None else geom.wire_arc[w][-1] / 2.0 for w, a, _v in self.feeds]
        if self.feeds and self.feed_smoothing_factor is None and self.feed_model == "point":
            # all point feeds in one batched evaluation: v_m = Phi_m(s_f)
            d = self.degree
            vals, first = T.point_values(basis.knots, d, ws, sfs)
            wi = np.repeat(np.asarray(ws, dtype=np.int64), d + 1)
            mg = basis.kept.global_index(wi, (first[:, None] + np.arange(d + 1)[None, :]).ravel())
            keep = (mg >= 0) & (vals.ravel() != 0.0)
            rs.append(mg[keep])
            cs.append(np.repeat(np.arange(len(ws), dtype=np.int64), d + 1)[keep])
            vs.append(vals.ravel()[keep].astype(np.complex128))
        else:
            for i, (w, s_f) in enumerate(zip(ws, sfs)):
                idx, val = self._source_entries(w, s_f)
                rs.append(idx)
                cs.append(np.full(idx.size, i, dtype=np.int64))
                vs.append(val)
        _kcl, port_A, _pv = self._split_kcl_ports(basis.kcl_A)
        pa = port_A.tocoo()
        rs.append(pa.col.astype(np.int64))
        cs.append(pa.row.astype(np.int64) + len(self.feeds))
        vs.append(pa.data.astype(np.complex128))
        gap, _gv = self._node_gap_columns()
        gr, gc = np.nonzero(gap)
        rs.append(gr.astype(np.int64))
        cs.append(gc.astype(np.int64) + len(self.feeds) + port_A.shape[0])
        vs.append(gap[gr, gc].astype(np.complex128))
        n_p = len(self.feeds) + port_A.shape[0] + gap.shape[1]
        return np.concatenate(rs), np.concatenate(cs), np.concatenate(vs), n_p

    def _port_count(self):
        return len(self.feeds) + len(self.junction_ports) + len(self.node_gaps)

    # ----------------------------------------------------------- device
    def _ground_struct(self):
        if self.ground_z is None:
            return None
        g = _lib.Ground()
        g.ground_z = float(self.ground_z)
        if self.ground_eps is None:
            g.model = _lib.MW_GROUND_PEC
            return g
        et = T.eps_tilde(self.ground_eps, self.omega, self.eps)
        g.eps_re, g.eps_im = et.real, et.imag
        if self.ground_model == "sommerfeld":
            g.model = _lib.MW_GROUND_SOMM_IMAGE  # C2 = (eps~-1)/(eps~+1) image
            return g
        g.model = _lib.MW_GROUND_REFL
        g.phi_mode = _lib.PHI_MODES[self.ground_phi_mode]
        return g

    def _alloc(self, enrich=None):
        """Device buffers of one solve at this geometry (reused across calls
        by the benchmark): Z, the same-edge table, the port right-hand sides
        [B | kcl_con^T], the sparse B^T and kcl_con (CSR), LU workspace,
        pivots, status and Y.  With ``enrich`` (enrichment specs) the system
        is the augmented one: the enrichment bases follow the polynomial
        ones, with zero port and KCL entries (``bspline.py:4150-4175``)."""
        torch = _torch()
        dev = self._torch_device()
        dt = self._dev_tables()
        n_poly = self._basis().n
        n = n_poly + (len(enrich) if enrich else 0)
        nm = self.degree + 1
        # port columns and KCL rows are a few nonzeros each: upload them in
        # coordinate form and scatter [B | kcl_con^T], B and kcl_con on the
        # device
        pr, pc, pv, n_p = self._port_entries()
        kcl_con = self._split_kcl_ports(self._basis().kcl_A)[0].tocoo()
        n_c = kcl_con.shape[0]
        kr, kc = kcl_con.row.astype(np.int64), kcl_con.col.astype(np.int64)
        kv = kcl_con.data.astype(np.complex128)
        rr, rc, rv = np.concatenate([pr, kc]), np.concatenate([pc, kr + n_p]), np.concatenate([pv, kv])
        # CSR of B^T (one row per port) and of kcl_con for the sparse
        # products Y = B^T X, A Xc and A W
        bt_ptr, bt_col, bt_val = _csr(pc, pr, pv, n_p)
        a_ptr, a_col, a_val = _csr(kr, kc, kv, n_c)
        host = [pr, pc, np.ascontiguousarray(pv).view(np.float64), kr, kc, np.ascontiguousarray(kv).view(np.float64),
                rr, rc, np.ascontiguousarray(rv).view(np.float64), bt_ptr, bt_col, bt_val.view(np.float64), a_ptr,
                a_col, a_val.view(np.float64)]
        # one page-locked staging buffer and one stream-ordered copy for all
        # of them (each array 256-byte aligned), device views by offset
        host = [np.ascontiguousarray(a) for a in host]
        offs, tot = [], 0
        for a in host:
            offs.append(tot)
            tot += (a.nbytes + 255) & ~255
        stage = torch.empty(max(tot, 256), dtype=torch.uint8, pin_memory=True)
        sv = stage.numpy()
        for a, o in zip(host, offs):
            sv[o:o + a.nbytes] = a.reshape(-1).view(np.uint8)
        dbytes = torch.empty(stage.numel(), dtype=torch.uint8, device=dev)
        dbytes.copy_(stage, non_blocking=True)
        tdt = {np.dtype(np.int64): torch.int64, np.dtype(np.float64): torch.float64}
        ent = [dbytes[o:o + a.nbytes].view(tdt[a.dtype]) for a, o in zip(host, offs)]
        lib = _lib.load()
        st = torch.cuda.current_stream(dev).cuda_stream
        m = n_p + n_c
        rhs0 = torch.empty((max(m, 1), n), dtype=torch.complex128, device=dev)
        _lib.call("mw_scatter_c128", n, m, rr.size, ent[6].data_ptr(), ent[7].data_ptr(), ent[8].data_ptr(),
                  rhs0.data_ptr(), st)
        buf = {
            "n": n,
            "n_poly": n_poly,
            "enrich": enrich or [],
            "n_p": n_p,
            "n_c": n_c,
            "Z": torch.empty((n, n), dtype=torch.complex128, device=dev),
            "table": torch.empty((max(dt.table_rows, 1), nm, nm), dtype=torch.complex128, device=dev),
            # column-major (n x m) right-hand sides live in an (m, n) tensor
            "RHS0": rhs0,
            "entries": ent,
            "ws": torch.empty(lib.mw_getrf_workspace_size(n), dtype=torch.uint8, device=dev),
            "ipiv": torch.empty(max(n, 1), dtype=torch.int32, device=dev),
            "info": torch.zeros(2, dtype=torch.int32, device=dev),
            "Y": torch.empty((max(n_p, 1), max(n_p, 1)), dtype=torch.complex128, device=dev),
            "kcl": kcl_con,
            "_stage": stage,  # the staging buffer lives until the copy has run
        }
        buf["RHS"] = torch.empty_like(buf["RHS0"])
        if self.precision == "mixed":
            m = n_p + n_c
            buf["Z32"] = torch.empty((n, n), dtype=torch.complex64, device=dev)
            buf["ws_mix"] = torch.empty(lib.mw_zgesv_mixed_workspace_size(n, m), dtype=torch.uint8, device=dev)
        if n_c:
            buf["S"] = torch.empty((n_c, n_c), dtype=torch.complex128, device=dev)
            buf["AW"] = torch.empty((max(n_p, 1), n_c), dtype=torch.complex128, device=dev)
            buf["ws_c"] = torch.empty(lib.mw_getrf_workspace_size(n_c), dtype=torch.uint8, device=dev)
            buf["ipiv_c"] = torch.empty(n_c, dtype=torch.int32, device=dev)
            buf["info_c"] = torch.zeros(2, dtype=torch.int32, device=dev)
            buf["W"] = torch.empty((max(n_p, 1), n), dtype=torch.complex128, device=dev)
        buf["h2d_bytes"] = int(sum(a.nbytes for a in host) + dt.h2d_bytes)
        return buf

    def _fill_device(self, buf, stream):
        """Fill buf["Z"] (complex128, column-major) at the current k."""
        dt = self._dev_tables()
        d = self.degree
        n = buf["n"]
        table = buf["table"]
        _lib.call("mw_same_edge_table", C.byref(dt.edges), d, self.n_qp_pair, int(self.extended_kernel),
                  float(self.k), table.data_ptr(), stream)
        fr = _lib.Freq(float(self.k), float(self.omega), float(self.eps), float(self.mu))
        Z = buf["Z"]
        z32 = buf["Z32"].data_ptr() if "Z32" in buf else None
        _lib.call("mw_fill_z", C.byref(dt.seg), C.byref(dt.basis), table.data_ptr(), C.byref(dt.edges),
                  C.byref(fr), self.n_qp_pair, Z.data_ptr(), n, z32, n, stream)
        g = self._ground_struct()
        if g is not None:
            _lib.call("mw_fill_z_image", C.byref(dt.seg), C.byref(dt.basis), C.byref(g), C.byref(fr),
                      self.n_qp_pair, Z.data_ptr(), n, z32, n, stream)
        if self._is_sommerfeld():
            use, info = self._surrogate_check(stream) if self.sommerfeld_method == "surrogate" else (None, {})
            if use is not None:
                feats = np.ascontiguousarray(info.pop("struct_features"), dtype=np.float32)
                vscale = sur.SCALE * (self.omega * self.mu) / (sur.OMEGA_REF * sur.MU0_GRID)
                _lib.call("mw_somm_remainder_q_mlp", C.byref(dt.seg), C.byref(dt.basis), use.pbf.data_ptr(),
                          use.p32.data_ptr(), feats.ctypes.data, float(self.wavelength), float(vscale),
                          self.n_qp_sommerfeld, float(self.ground_z), float(self.k), Z.data_ptr(), n, z32, n,
                          use.err.data_ptr(), stream)
                self.last_sommerfeld = dict(info, method="surrogate")
            else:
                grid = self._somm_grid(stream)
                _lib.call("mw_somm_remainder_q", C.byref(dt.seg), C.byref(dt.basis), C.byref(grid),
                          self.n_qp_sommerfeld, float(self.ground_z), float(self.k), Z.data_ptr(), n, z32, n, stream)
                self.last_sommerfeld = dict(info, method="grid")
        # distributed series wire loading, added once to the final Z
        self._loading_device(Z, buf.get("Z32"), [self.omega], stream)
        if buf["enrich"]:
            self._enrich_device(buf, stream)

    # ----------------------------------------------------------- enrichment
    def _enrich_device(self, buf, stream):
        """The enrichment blocks of the augmented Z (and Z32): quadrature on
        the device (``mw_enrich_blocks``), the Sommerfeld remainder reaction
        from device field projections, and the "tikhonov" variant's
        lambda * mean|diag Z_ee| on the enrichment diagonal
        (``bspline.py:3523-3693``, ``4162-4164``)."""
        torch = _torch()
        dev = buf["Z"].device
        sp = buf["enrich"]
        n, n_poly, E = buf["n"], buf["n_poly"], len(sp)
        dt = self._dev_tables()
        t, w = EN.gauss01(self.n_qp_sing)
        poly = EN.shape_polynomial(self.enrichment_variant, self.degree)
        seg = torch.tensor([s.seg for s in sp], dtype=torch.int32, device=dev)
        org = torch.tensor([s.origin for s in sp], dtype=torch.int32, device=dev)
        t_d = torch.from_numpy(t).to(dev)
        w_d = torch.from_numpy(w).to(dev)
        en = _lib.Enrich()
        en.n_enrich, en.seg, en.origin, en.n_qp = E, seg.data_ptr(), org.data_ptr(), int(self.n_qp_sing)
        en.t01, en.w01 = t_d.data_ptr(), w_d.data_ptr()
        for i in range(4):
            en.proj[i] = float(poly[i]) if i < poly.size else 0.0
        en.radius = float(self._radius_per_wire[0])
        fr = _lib.Freq(float(self.k), float(self.omega), float(self.eps), float(self.mu))
        g = self._ground_struct()
        Z = buf["Z"]
        Z32 = buf.get("Z32")
        _lib.call("mw_enrich_blocks", C.byref(dt.seg), C.byref(dt.basis), C.byref(en), C.byref(fr),
                  C.byref(g) if g is not None else None, Z.data_ptr(), n,
                  Z32.data_ptr() if Z32 is not None else None, n, stream)
        # column-major Z in a row-major (n, n) tensor: Z[row, col] is zt[col, row]
        zt = Z.view(n, n)
        if self._is_sommerfeld():
            q_pe, q_ee = self._enrich_somm_remainder(sp, t, w, poly, stream)
            zt[n_poly:, :n_poly] -= q_pe.T  # Z_pe (rows m, columns e)
            zt[:n_poly, n_poly:] -= q_pe  # Z_ep = Z_pe^T by reciprocity
            zt[n_poly:, n_poly:] -= q_ee.T
        if self.enrichment_variant == "tikhonov":
            d = torch.diagonal(zt[n_poly:, n_poly:])
            scale = float(self.tikhonov_lambda) * float(d.abs().mean())
            d += scale
        if Z32 is not None and (self._is_sommerfeld() or self.enrichment_variant == "tikhonov"):
            z32t = Z32.view(n, n)
            z32t[n_poly:, :] = zt[n_poly:, :].to(torch.complex64)
            z32t[:n_poly, n_poly:] = zt[:n_poly, n_poly:].to(torch.complex64)

    def _enrich_somm_remainder(self, sp, t, w, poly, stream):
        """(Q_pe (n_poly, E), Q_ee (E, E)): the Sommerfeld remainder field
        between the enrichment bases' nodes (weight times shape) and the
        polynomial bases' n_qp_sommerfeld nodes per segment (u^p moments
        contracted with the basis polynomials), ``bspline.py:1919-2033``.
        Field projections on the device (mw_somm_field_proj), contractions
        as device GEMMs."""
        torch = _torch()
        dev = self._torch_device()
        geom, basis = self._geometry(), self._basis()
        grid = self._somm_grid(stream)
        E, q_e = len(sp), t.size
        pts_e, val_e = EN.shape_values(sp, geom, t, poly)
        h_e = np.array([geom.h[s.seg] for s in sp])
        wphi = torch.from_numpy((w[None, :] * h_e[:, None]) * val_e).to(dev).to(torch.complex128)  # (E, q_e)
        obs_e = torch.from_numpy(np.ascontiguousarray(pts_e.reshape(-1, 3))).to(dev)
        tan_e = torch.from_numpy(np.ascontiguousarray(np.repeat(geom.tangents[[s.seg for s in sp]], q_e, 0))).to(dev)
        q = int(self.n_qp_sommerfeld)
        tq, wq = EN.gauss01(q)
        nodes = geom.seg_l[:, None, :] + tq[None, :, None] * (geom.seg_r - geom.seg_l)[:, None, :]
        obs_p = torch.from_numpy(np.ascontiguousarray(nodes.reshape(-1, 3))).to(dev)
        tan_p = torch.from_numpy(np.ascontiguousarray(np.repeat(geom.tangents, q, axis=0))).to(dev)
        n_seg, d1 = geom.n, self.degree + 1

        def proj(o, to, s_, ts):
            out = torch.empty((o.shape[0], s_.shape[0]), dtype=torch.complex128, device=dev)
            _lib.call("mw_somm_field_proj", o.shape[0], o.data_ptr(), to.data_ptr(), s_.shape[0], s_.data_ptr(),
                      ts.data_ptr(), float(self.ground_z), float(self.k), C.byref(grid), out.data_ptr(), stream)
            return out

        f_ee = proj(obs_e, tan_e, obs_e, tan_e).view(E, q_e, E, q_e)
        q_ee = torch.einsum("eq,eqfr,fr->ef", wphi, f_ee, wphi)
        f_pe = proj(obs_p, tan_p, obs_e, tan_e).view(n_seg, q, E, q_e)
        field = torch.einsum("iqer,er->iqe", f_pe, wphi)  # (n_seg, q, E)
        u = geom.h[:, None] * tq[None, :]
        wm = (wq[None, :] * geom.h[:, None])[None] * u[None] ** np.arange(d1)[:, None, None]
        jf = torch.einsum("piq,iqe->pie", torch.from_numpy(wm).to(dev).to(torch.complex128), field)  # (d1, n_seg, E)
        supp = torch.from_numpy(basis.supp.astype(np.int64)).to(dev)
        polys = torch.from_numpy(basis.polys).to(dev).to(torch.complex128)
        q_pe = torch.zeros((basis.n, E), dtype=torch.complex128, device=dev)
        for a in range(d1):
            sm = supp[:, a].clamp(min=0)
            live = (supp[:, a] >= 0).to(torch.complex128)[:, None]
            q_pe += live * torch.einsum("mp,pme->me", polys[:, a, :], jf[:, sm, :])
        return q_pe, q_ee

    # ------------------------------------------------------------ loading
    def _loading_tables(self) -> wl.LoadingGram:
        if self._cached_loading is None:
            self._cached_loading = wl.loading_gram(self._geometry(), self._basis())
        return self._cached_loading

    def _loading_gram(self):
        """(rows, cols, vals, wire_of_nnz) triplets of the same-wire
        basis-overlap Gram, one per shared segment (``bspline.py:2667-2731``)."""
        g = self._loading_tables()
        return g.rows, g.cols, g.vals, g.wire

    def _apply_loading(self, Z, omega=None):
        """Add the loading term into a host Z (n, n) or stack (n_k, n, n) in
        place; a no-op when no loading is configured (``bspline.py:2732-2760``).
        The device fill applies the same term through ``mw_add_loading``."""
        if self._loading is None:
            return Z
        g = self._loading_tables()
        zw = self._loading.z_wire(self.omega if omega is None else omega)
        if Z.ndim == 2:
            np.add.at(Z, (g.rows, g.cols), zw[g.wire] * g.vals)
        else:
            data = zw[g.wire, :].T * g.vals[None, :]
            for ki in range(Z.shape[0]):
                np.add.at(Z[ki], (g.rows, g.cols), data[ki])
        return Z

    def wire_loss_power(self, coeffs, omega=None):
        """Ohmic power in the wire metal from a solve's coefficients:
        P = 1/2 sum_w Re Z'_w (c^H S_w c); returns (total W, per-wire W)
        (``bspline.py:2782-2806``).  Insulation is reactive and adds nothing."""
        per_wire = np.zeros(len(self.wires_polylines), dtype=np.float64)
        if self._loading is None:
            return 0.0, per_wire
        g = self._loading_tables()
        c = np.asarray(coeffs)[: self._basis().n]
        r_w = np.real(self._loading.z_wire(self.omega if omega is None else omega))
        contrib = 0.5 * r_w[g.wire] * np.real(np.conj(c[g.rows]) * c[g.cols]) * g.vals
        np.add.at(per_wire, g.wire, contrib)
        return float(per_wire.sum()), per_wire

    def _loading_dev_tables(self):
        """Device copies of the coalesced Gram entries (rows, cols, vals,
        wire), uploaded once per solver; None without loading."""
        if self._loading is None:
            return None
        if self._cached_loading_dev is None:
            torch = _torch()
            dev = self._torch_device()
            g = self._loading_tables()
            self._cached_loading_dev = (
                torch.from_numpy(g.u_rows.astype(np.int64)).to(dev),
                torch.from_numpy(g.u_cols.astype(np.int64)).to(dev),
                torch.from_numpy(g.u_vals.astype(np.float64)).to(dev),
                torch.from_numpy(g.u_wire.astype(np.int32)).to(dev),
            )
        return self._cached_loading_dev

    def _loading_device(self, Z, Z32, omegas, stream, ld=None):
        """Z_b += sum_w Z'_w(omega_b) S_w on the device for a stack of
        column-major matrices (Z: (n_k, ld, ld) or (ld, ld) tensor, ld = n
        by default; Z32 its complex64 mirror or None)."""
        if self._loading is None:
            return
        torch = _torch()
        dev = self._torch_device()
        n = self._basis().n
        rows, cols, vals, wire = self._loading_dev_tables()
        omegas = np.atleast_1d(np.asarray(omegas, dtype=np.float64))
        zw = np.ascontiguousarray(self._loading.z_wire(omegas).T)  # (batch, n_wires)
        zh = torch.empty(zw.shape, dtype=torch.complex128, pin_memory=True)
        zh.copy_(torch.from_numpy(zw))
        zt = zh.to(dev, non_blocking=True)
        batch = omegas.size
        ld = n if ld is None else int(ld)
        _lib.call("mw_add_loading", n, batch, rows.numel(), rows.data_ptr(), cols.data_ptr(), vals.data_ptr(),
                  wire.data_ptr(), zt.data_ptr(), zw.shape[1], Z.data_ptr(), ld, ld * ld,
                  Z32.data_ptr() if Z32 is not None else None, ld, ld * ld, None, stream)

    def _surrogate_check(self, stream):
        """(model, info) when the surrogate may serve this structure at this
        k, else (None, info with the reason): the weights must exist, eps~
        and f and every Gauss-node pair must lie in the training domain, and
        the largest error of a quadrature spot check on sampled node pairs,
        relative to the largest quadrature surface value, must be within
        ``surrogate_tol``."""
        model = sur.get_model(self._torch_device())
        if model is None:
            return None, {"reason": "no surrogate weights"}
        et = complex(T.eps_tilde(self.ground_eps, self.omega, self.eps))
        f = self.omega / (2.0 * np.pi)
        lam = self.wavelength
        geom = self._geometry()
        q = self.n_qp_sommerfeld
        tq = 0.5 * (np.polynomial.legendre.leggauss(q)[0] + 1.0)
        nodes = (geom.seg_l[:, None, :] + tq[None, :, None] * (geom.seg_r - geom.seg_l)[:, None, :]).reshape(-1, 3)
        zmin = float(nodes[:, 2].min()) - self.ground_z
        r1_max = float(somm.max_image_distance(self._dev_tables().seg.seg_l, self._dev_tables().seg.seg_r,
                                               self._dev_tables().seg.n_seg, self.ground_z, self._torch_device(),
                                               stream)) / 1.001
        ok = sur.in_domain(np.array([0.0, 0.0]), np.array([2.0 * zmin / lam, sur.H_MIN_WL]), np.array([et, et]),
                           np.array([f, f]))
        if not (ok.all() and r1_max / lam <= sur.R1_MAX_WL):
            return None, {"reason": "outside the surrogate domain"}
        rng = np.random.default_rng(1234)
        a = rng.integers(0, nodes.shape[0], sur.SPOT_PAIRS)
        b = rng.integers(0, nodes.shape[0], sur.SPOT_PAIRS)
        d = nodes[a] - nodes[b]
        rho = np.hypot(d[:, 0], d[:, 1]) / lam
        h = ((nodes[a, 2] - self.ground_z) + (nodes[b, 2] - self.ground_z)) / lam
        err, rel = sur.spot_check(model, rho, h, et, f)
        info = {"spot_max_err": err, "spot_rel_err": rel, "struct_features": sur.features(0.0, 1.0, et, f)[2:5]}
        if not rel <= self.surrogate_tol:
            info.pop("struct_features")
            info["reason"] = f"spot check {rel:.2e} over surrogate_tol {self.surrogate_tol:.1e}"
            return None, info
        return model, info

    def _is_sommerfeld(self):
        return self.ground_z is not None and self.ground_eps is not None and self.ground_model == "sommerfeld"

    def _somm_grid(self, stream):
        """``mw_somm_grid`` of the remainder grid at the current k
        (``bspline.py:1781-1789``, ``:1859-1862``): the cached
        wavelength-normalised master for (bucketed eps~, r1 bucket), viewed
        at this k, omega and mu."""
        dt = self._dev_tables()
        dev = self._torch_device()
        if getattr(self, "_somm_r1", None) is None:
            self._somm_r1 = somm.max_image_distance(dt.seg.seg_l, dt.seg.seg_r, dt.seg.n_seg, self.ground_z, dev,
                                                    stream)
        et = T.eps_tilde(self.ground_eps, self.omega, self.eps)
        master = somm.get_master(et, self.k, self._somm_r1, dev, stream)
        self._somm_master = master
        return master.view(self.k, self.omega, self.mu)

    def _lu_solve(self, A, n, ws, ipiv, info, rhs, nrhs, stream):
        """zgetrf(A) in place then zgetrs on rhs (both column-major, ld n)."""
        cancel = C.c_void_p(self._cancel.ptr) if self._cancel is not None else None
        try:
            _lib.call("mw_zgetrf", n, A.data_ptr(), n, ipiv.data_ptr(), info.data_ptr(), ws.data_ptr(),
                      ws.numel(), cancel, stream)
        except _lib.NativeError as e:
            if e.status == _lib.MW_ERR_CANCELLED:
                raise SolveAborted() from e
            raise
        if nrhs:
            _lib.call("mw_zgetrs", n, nrhs, A.data_ptr(), n, ipiv.data_ptr(), rhs.data_ptr(), n, stream)

    def _device_solve(self, buf, stream):
        """The whole device pipeline of compute_port_solution: fill, LU,
        solve all port columns, KCL Schur step, Y = B^T X.  Returns the
        device tensor holding X (column-major, n x n_p)."""
        n, n_p, n_c = buf["n"], buf["n_p"], buf["n_c"]
        self._fill_device(buf, stream)
        if self.precision == "mixed":
            # complex64 tensor-core LU + FP64 refinement against Z
            m = n_p + n_c
            it, corr = C.c_int32(0), C.c_double(0.0)
            cancel = C.c_void_p(self._cancel.ptr) if self._cancel is not None else None
            try:
                _lib.call("mw_zgesv_mixed", n, m, buf["Z"].data_ptr(), n, buf["Z32"].data_ptr(), n,
                          buf["ipiv"].data_ptr(), buf["RHS0"].data_ptr(), n, buf["RHS"].data_ptr(), n,
                          float(self.mixed_tol), int(self.mixed_max_iter), buf["ws_mix"].data_ptr(),
                          buf["ws_mix"].numel(), buf["info"].data_ptr(), C.byref(it), C.byref(corr), cancel, stream)
            except _lib.NativeError as e:
                if e.status == _lib.MW_ERR_CANCELLED:
                    raise SolveAborted() from e
                raise
            self.last_refinement = {"iterations": int(it.value), "last_correction": float(corr.value)}
        else:
            buf["RHS"].copy_(buf["RHS0"], non_blocking=True)
            self._lu_solve(buf["Z"], n, buf["ws"], buf["ipiv"], buf["info"], buf["RHS"], n_p + n_c, stream)
        X = buf["RHS"]
        ent = buf["entries"]
        if n_c:
            # Lam = (A Xc)^-1 (A W); X <- W - Xc Lam   (bspline.py:2980-2989);
            # A (the KCL rows, a few +-1 each) applied as a sparse gather
            S, AW = buf["S"], buf["AW"]
            Wd, Xc = X[:n_p], X[n_p:]
            _lib.call("mw_csr_mm_c128", n_c, n_c, ent[12].data_ptr(), ent[13].data_ptr(), ent[14].data_ptr(),
                      Xc.data_ptr(), n, S.data_ptr(), n_c, stream)
            if n_p:
                _lib.call("mw_csr_mm_c128", n_c, n_p, ent[12].data_ptr(), ent[13].data_ptr(), ent[14].data_ptr(),
                          Wd.data_ptr(), n, AW.data_ptr(), n_c, stream)
            self._lu_solve(S, n_c, buf["ws_c"], buf["ipiv_c"], buf["info_c"], AW, n_p, stream)
            W = buf["W"][:n_p]
            W.copy_(Wd, non_blocking=True)
            if n_p:
                _lib.call("mw_zgemm", 0, 0, n, n_p, n_c, -1.0, 0.0, Xc.data_ptr(), n, AW.data_ptr(), n_c, 1.0,
                          0.0, W.data_ptr(), n, stream)
            X = W
        if n_p:
            # Y = B^T X with B's few nonzeros per port column
            _lib.call("mw_csr_mm_c128", n_p, n_p, ent[9].data_ptr(), ent[10].data_ptr(), ent[11].data_ptr(),
                      X.data_ptr(), n, buf["Y"].data_ptr(), n_p, stream)
        return X

    def _check_info(self, buf, infos=None):
        """Raise on a singular factor or a timed-out panel barrier; ``infos``
        are host copies of the status words already read back, if any."""
        if infos is None:
            infos = [buf["info"]] + ([buf["info_c"]] if buf["n_c"] else [])
            infos = [inf.cpu().numpy() for inf in infos]
        for v in infos:
            if v[1] != 0:
                raise RuntimeError(f"LU panel barrier timed out (device status {int(v[1])})")
            if v[0] > 0:
                raise np.linalg.LinAlgError("Matrix is singular.")

    def _compute_Z_operator(self, *_unused):
        """Host copy of Z (numpy complex128) -- for tests and for callers of
        the reference's private helper of the same name."""
        torch = _torch()
        buf = self._alloc()
        st = torch.cuda.current_stream(buf["Z"].device).cuda_stream
        self._fill_device(buf, st)
        return buf["Z"].cpu().numpy().T.copy()

    def compute_port_solution(self, same_edge_prep=None) -> PortSolution:
        """Solve every port from ONE fill and ONE factorisation
        (``bspline.py:4053-4179``).  ``same_edge_prep`` (the reference's
        precomputed same-edge moments for sweeps) is accepted for signature
        compatibility and unused: the device builds its same-edge table at
        each call for a fraction of a millisecond.

        With ``use_singular_enrichment`` the system is augmented by the
        enrichment bases (coefficients after the polynomial ones); the
        "auto" variant first solves without them and enriches only the
        junctions whose tap ratio exceeds ``auto_tap_ratio_threshold`` under
        any port's drive (``bspline.py:4121-4175``)."""
        self._checkpoint()
        self._auto_active_junctions = None
        enrich = None
        if self.use_singular_enrichment:
            active = None
            if self.enrichment_variant == "auto":
                first = self._solve_once(None)
                act = set()
                for j in range(first.coeffs.shape[1]):
                    cur = self.currents_at_knots(first.coeffs[:, j])
                    act |= {i for i, r in enumerate(EN.tap_ratios(self.junctions, cur, self.enrichment_min_k))
                            if r is not None and r > self.auto_tap_ratio_threshold}
                active = sorted(act)
                self._auto_active_junctions = active
                if not active:
                    return first
            enrich = EN.specs(self.junctions, self._geometry(), self.enrichment_min_k, active) or None
        return self._solve_once(enrich)

    def _enrichment_specs_now(self):
        """The enrichment bases of the last solve's system (empty when off)."""
        if not self.use_singular_enrichment:
            return []
        return EN.specs(self.junctions, self._geometry(), self.enrichment_min_k, self._auto_active_junctions)

    def _solve_once(self, enrich) -> PortSolution:
        torch = _torch()
        geom, basis = self._geometry(), self._basis()
        buf = self._alloc(enrich)
        st = torch.cuda.current_stream(buf["Z"].device).cuda_stream
        X = self._device_solve(buf, st)
        n_p = buf["n_p"]
        # one stream-ordered read-back into page-locked host memory: the
        # coefficients stay column-major (Xh is the transposed view), Y and
        # the status words ride along, then a single stream synchronise
        dev_stream = torch.cuda.current_stream(buf["Z"].device)
        hx = torch.empty(X.shape, dtype=X.dtype, pin_memory=True)
        hx.copy_(X, non_blocking=True)
        hy = torch.empty((n_p, n_p), dtype=X.dtype, pin_memory=True)
        if n_p:
            hy.copy_(buf["Y"][:n_p, :n_p], non_blocking=True)
        hinfo = [torch.empty(2, dtype=torch.int32, pin_memory=True)
                 for _ in range(2 if buf["n_c"] else 1)]
        hinfo[0].copy_(buf["info"][:2], non_blocking=True)
        if buf["n_c"]:
            hinfo[1].copy_(buf["info_c"][:2], non_blocking=True)
        dev_stream.synchronize()
        Xh = hx.numpy().T
        Yh = hy.numpy().T
        self._check_info(buf, [h.numpy() for h in hinfo])
        self.last_stats = {"h2d_bytes": buf["h2d_bytes"], "d2h_bytes": int(Xh.nbytes + Yh.nbytes + 16)}
        return PortSolution(
            y=Yh,
            coeffs=Xh,
            port_currents=Yh,
            basis=_SplineBasis(geom, basis.supp, basis.polys, basis.knots, basis.kept, basis.n),
        )

    def compute_y_matrix(self) -> np.ndarray:
        """Short-circuit admittance matrix (``bspline.py:4019``)."""
        return self.compute_port_solution().y

    def compute_impedance(self, same_edge_prep=None):
        """Drive-point impedance(s) for the configured voltages and the
        solved coefficients (``bspline.py:3919-4017``)."""
        sol = self.compute_port_solution()
        _kcl, _pa, port_V = self._split_kcl_ports(self._basis().kcl_A)
        _gap, gap_V = self._node_gap_columns()
        volts = np.concatenate([np.array([v for _w, _a, v in self.feeds], dtype=np.complex128), port_V, gap_V])
        coeffs = sol.coeffs @ volts
        pr, pc, pv, n_p = self._port_entries()
        nb = self._basis().n
        Bs = scipy.sparse.csr_matrix((pv, (pr, pc)), shape=(nb, n_p))
        currents = Bs.T @ coeffs[:nb]  # port entries sit on the polynomial bases
        z = volts / currents
        return (z[0] if len(volts) == 1 else z), coeffs

    # --------------------------------------------------------------- sweeps
    def compute_port_solution_swept(self, k_array):
        """One ``PortSolution`` per wavenumber (``_port_solution.py:127``)."""
        out = []
        with self._k_restored():
            for kk in np.asarray(k_array, dtype=float):
                self._checkpoint()
                self._set_k(kk)
                out.append(self.compute_port_solution())
        return out

    def compute_y_matrix_swept(self, k_array) -> np.ndarray:
        """(n_k, n_ports, n_ports) Y matrices (``_port_solution.py:142``).

        On free space or a PEC ground every frequency of a chunk is filled in
        one batched launch; with ``precision="mixed"`` the chunk is then
        factorised together (``_swept_batched``), with ``"fp64"`` each
        matrix of the stack takes the complex128 LU (``_swept_fp64_batched``,
        the reference's k-batched fill with stacked LAPACK solves).  KCL
        constraint rows (junctions) ride along as extra right-hand sides and
        the Schur step closes each frequency (``bspline.py:3017-3038``).
        Other grounds take the single-solve path per k."""
        k_array = np.asarray(k_array, dtype=float)
        self._checkpoint()
        if k_array.shape[0] == 0:
            n_p = self._port_count()
            return np.zeros((0, n_p, n_p), dtype=np.complex128)
        if self._swept_batched_available():
            return self._swept_batched(k_array)
        if self._swept_fp64_batched_available():
            return self._swept_fp64_batched(k_array)
        n_p = self._port_count()
        out = np.zeros((k_array.shape[0], n_p, n_p), dtype=np.complex128)
        for i, sol in enumerate(self.compute_port_solution_swept(k_array)):
            out[i] = sol.y
        return out

    # KCL rows a batched sweep carries as extra right-hand sides
    SWEPT_MAX_KCL = 64

    def _swept_batched_available(self):
        """Batched mixed route: mixed precision, free space or PEC image
        (finite grounds carry per-k weight tables), at most SWEPT_MAX_KCL
        KCL rows left after the port split, order within the batched
        panel's limit."""
        if self.precision != "mixed" or self.ground_eps is not None or self.use_singular_enrichment:
            return False
        return self._kcl_rows_left() <= self.SWEPT_MAX_KCL and self._basis_count() <= 1600

    def _swept_fp64_batched_available(self):
        """Batched-fill FP64 route: complex128, free space or PEC image, at
        most SWEPT_MAX_KCL KCL rows."""
        return (self.precision == "fp64" and self.ground_eps is None and not self.use_singular_enrichment
                and self._kcl_rows_left() <= self.SWEPT_MAX_KCL)

    def _sweep_rhs(self):
        """(R, B, A): the right-hand sides of a swept solve, R = [B | A^T]
        (n x (P + n_c), complex128) with B the port columns and A the dense
        KCL constraint rows (n_c x n)."""
        B, kcl = self._port_columns()
        A = kcl.toarray().astype(np.complex128) if kcl.shape[0] else np.zeros((0, B.shape[0]), np.complex128)
        return np.hstack([B, A.T]), B, A

    def _basis_count(self):
        """Order of the system without building the basis: per wire its
        segments + d - 2 interior bases plus the end bases a junction or the
        ground holds (the rule of ``_tables.build_basis``)."""
        if self._cached_basis is not None:
            return self._basis().n
        held = int(np.count_nonzero(self._end_table() != topo.FREE))
        segs = sum(sum(npe) for npe in self.n_per_edge_per_wire)
        return int(segs + (self.degree - 2) * len(self.n_per_edge_per_wire) + held)

    def _kcl_rows_left(self):
        """KCL constraint rows that stay after the junction-port split: one
        per junction off the ground, less the junction ports."""
        grounded = self._grounded_junctions()
        return sum(1 for j in range(len(self.junctions)) if j not in grounded) - len(self.junction_ports)

    def _fill_batched(self, ks, stream, Z=None, Z32=None, ld=None, k_dev=None, want32=True):
        """(Z, Z32): device (n_k, n, n) complex128 / complex64 stacks, each
        matrix column-major (Z[b].T is the matrix at ks[b]), from one
        batched fill launch.  Given Z / Z32 of shape (n_k, ld, ld) with
        ld >= n, the fill writes the leading n x n block of each.  k_dev:
        the (2, n_k) float64 device tensor [k; omega] when the caller has
        uploaded it already (a pageable upload would wait for the stream)."""
        torch = _torch()
        dev = self._torch_device()
        dt = self._dev_tables()
        n, d = self._basis().n, self.degree
        nk = len(ks)
        ld = n if ld is None else int(ld)
        if k_dev is None:
            k_dev = self._upload_k(ks)
        kb, ob = k_dev[0], k_dev[1]
        table = torch.empty((nk, max(dt.table_rows, 1), d + 1, d + 1), dtype=torch.complex128, device=dev)
        if Z is None:
            Z = torch.empty((nk, ld, ld), dtype=torch.complex128, device=dev)
        if Z32 is None and want32:
            Z32 = torch.empty((nk, ld, ld), dtype=torch.complex64, device=dev)
        pec = 1 if self.ground_z is not None else 0
        _lib.call("mw_fill_z_batch", C.byref(dt.seg), C.byref(dt.basis), C.byref(dt.edges), nk, kb.data_ptr(),
                  ob.data_ptr(), float(self.eps), float(self.mu), self.n_qp_pair, int(self.extended_kernel),
                  float(self.ground_z or 0.0), pec, table.data_ptr(), Z.data_ptr(), ld, ld * ld,
                  Z32.data_ptr() if Z32 is not None else None, ld, ld * ld, stream)
        self._loading_device(Z, Z32, np.asarray(ks, dtype=np.float64) * self.c, stream, ld=ld)
        return Z, Z32

    def _upload_k(self, ks):
        """[k; omega] (2, n_k) float64 on the device, through page-locked
        memory with a stream-ordered copy (no host wait on queued work)."""
        torch = _torch()
        h = torch.empty((2, len(ks)), dtype=torch.float64, pin_memory=True)
        h[0] = torch.from_numpy(np.asarray(ks, dtype=np.float64))
        h[1] = torch.from_numpy(np.asarray(ks, dtype=np.float64) * self.c)
        return h.to(self._torch_device(), non_blocking=True)

    def _batched_panel_width(self, ks):
        """Columns per batched panel step for this order: the autotuner's
        cached choice for (n bucket, degree, ground), timed on a short sweep
        of this structure the first time the bucket is met."""
        if getattr(self, "_panel_width", None):
            return self._panel_width
        torch = _torch()
        ground = "free" if self.ground_z is None else "pec"
        ks = np.asarray(ks, dtype=np.float64)
        probe = np.linspace(ks.min(), ks.max(), min(len(ks), 16))

        def time_width(w):
            self._panel_width = w
            try:
                self._swept_batched(probe)  # warm-up
                st = torch.cuda.current_stream(self._torch_device())
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(st)
                self._swept_batched(probe)
                b.record(st)
                b.synchronize()
                return a.elapsed_time(b)
            finally:
                self._panel_width = None

        self._panel_width = autotune.choose(self._basis().n, self.degree, ground, time_width)
        return self._panel_width

    def _swept_batched(self, k_array, mem_budget_bytes=16 << 30):
        """Chunked batched sweep: per chunk of frequencies, one batched fill
        (Z in complex128 and complex64) and one batched mixed solve with FP64
        refinement; Y_k = B^T X_k."""
        pw = self._batched_panel_width(k_array)
        torch = _torch()
        dev = self._torch_device()
        dt = self._dev_tables()
        basis = self._basis()
        n, d = basis.n, self.degree
        R, B, A = self._sweep_rhs()
        n_p = R.shape[1]
        per_k = n * n * (16 + 8) + dt.table_rows * (d + 1) ** 2 * 16 + n * n_p * 48 + n * 4
        chunk = int(max(1, min(len(k_array), 65535, mem_budget_bytes // max(per_k, 1))))
        st = torch.cuda.current_stream(dev).cuda_stream
        lib = _lib.load()
        Bh = torch.empty((n_p, n), dtype=torch.complex128, pin_memory=True)
        Bh.copy_(torch.from_numpy(np.ascontiguousarray(R.T)))
        Bd = Bh.to(dev, non_blocking=True)  # column-major n x (P + n_c)
        out = np.zeros((len(k_array), B.shape[1], B.shape[1]), dtype=np.complex128)
        iters = []
        for c0 in range(0, len(k_array), chunk):
            self._checkpoint()
            ks = np.asarray(k_array[c0 : c0 + chunk], dtype=np.float64)
            nk = len(ks)
            Z, Z32 = self._fill_batched(ks, st)
            X = torch.empty((nk, n_p, n), dtype=torch.complex128, device=dev)
            ipiv = torch.empty((nk, n), dtype=torch.int32, device=dev)
            info = torch.zeros(nk, dtype=torch.int32, device=dev)
            wsb = lib.mw_zgesv_mixed_batched_workspace_size(n, n_p, nk)
            ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
            it, corr = C.c_int32(0), C.c_double(0.0)
            _lib.call("mw_zgesv_mixed_batched", n, n_p, nk, int(pw), Z.data_ptr(), n,
                      n * n, Z32.data_ptr(), n, n * n,
                      ipiv.data_ptr(), info.data_ptr(), Bd.data_ptr(), n, 0, X.data_ptr(), float(self.mixed_tol),
                      int(self.mixed_max_iter), ws.data_ptr(), wsb, C.byref(it), C.byref(corr), st)
            iters.append(int(it.value))
            out[c0 : c0 + nk] = _swept_y(X.cpu().numpy(), B, A)  # X: (nk, P + n_c, n), X_k^T
            del Z, Z32, X, ws
        self.last_refinement = {"iterations": max(iters) if iters else 0, "chunks": len(iters)}
        return out

    def _swept_fp64_batched(self, k_array, mem_budget_bytes=16 << 30):
        """FP64 sweep: per chunk of frequencies one batched complex128 fill,
        then each matrix of the stack factorised and solved in complex128
        (``mw_zgetrf`` / ``mw_zgetrs``) on the device, the right-hand sides
        [B | A^T] uploaded once; Y_k from the Schur step on the host."""
        torch = _torch()
        dev = self._torch_device()
        dt = self._dev_tables()
        n, d = self._basis().n, self.degree
        R, B, A = self._sweep_rhs()
        m = R.shape[1]
        per_k = n * n * 16 + dt.table_rows * (d + 1) ** 2 * 16 + n * m * 16 + n * 4
        chunk = int(max(1, min(len(k_array), 65535, mem_budget_bytes // max(per_k, 1))))
        st = torch.cuda.current_stream(dev).cuda_stream
        lib = _lib.load()
        Rh = torch.empty((m, n), dtype=torch.complex128, pin_memory=True)
        Rh.copy_(torch.from_numpy(np.ascontiguousarray(R.T)))
        Rd = Rh.to(dev, non_blocking=True)  # column-major n x (P + n_c)
        wsb = lib.mw_getrf_workspace_size(n)
        ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
        cancel = C.c_void_p(self._cancel.ptr) if self._cancel is not None else None
        out = np.zeros((len(k_array), B.shape[1], B.shape[1]), dtype=np.complex128)
        for c0 in range(0, len(k_array), chunk):
            self._checkpoint()
            ks = np.asarray(k_array[c0 : c0 + chunk], dtype=np.float64)
            nk = len(ks)
            Z, _ = self._fill_batched(ks, st, want32=False)
            X = Rd.unsqueeze(0).repeat(nk, 1, 1)  # (nk, m, n): X_k^T, overwritten by the solves
            ipiv = torch.empty((nk, n), dtype=torch.int32, device=dev)
            info = torch.zeros((nk, 2), dtype=torch.int32, device=dev)
            for b in range(nk):
                try:
                    _lib.call("mw_zgetrf", n, Z[b].data_ptr(), n, ipiv[b].data_ptr(), info[b].data_ptr(),
                              ws.data_ptr(), wsb, cancel, st)
                except _lib.NativeError as e:
                    if e.status == _lib.MW_ERR_CANCELLED:
                        raise SolveAborted() from e
                    raise
                _lib.call("mw_zgetrs", n, m, Z[b].data_ptr(), n, ipiv[b].data_ptr(), X[b].data_ptr(), n, st)
            hinfo = info.cpu().numpy()
            if np.any(hinfo[:, 1] != 0):
                raise RuntimeError("factorisation: a bounded device wait timed out")
            if np.any(hinfo[:, 0] > 0):
                raise np.linalg.LinAlgError("Singular matrix")
            out[c0 : c0 + nk] = _swept_y(X.cpu().numpy(), B, A)
            del Z, X
        self.last_refinement = None
        return out

    def compute_impedance_swept(self, k_array):
        """Drive-point impedances over a batch of wavenumbers
        (``bspline.py:4479-4513``): complex, (n_k,) for one port and
        (n_k, n_feeds + n_junction_ports) otherwise -- the layout the
        reference allocates before its per-k loop, empty sweeps included."""
        k_array = np.asarray(k_array, dtype=float)
        n_total = len(self.feeds) + len(self.junction_ports)
        shape = (k_array.shape[0],) if n_total == 1 else (k_array.shape[0], n_total)
        z_out = np.zeros(shape, dtype=np.complex128)
        with self._k_restored():
            for i, kk in enumerate(k_array):
                self._checkpoint()
                self._set_k(kk)
                z_out[i] = self.compute_impedance()[0]
        return z_out

    # -------------------------------------------------------------- readout
    def currents_at_knots(self, coeffs, s_array=None):
        """Per-wire complex current at every mesh knot, or at the given arc
        positions (``bspline.py:4586-4685``)."""
        coeffs = np.asarray(coeffs)
        geom, basis = self._geometry(), self._basis()
        d = self.degree
        out = []
        for w in range(len(self.wires_polylines)):
            knots = basis.knots[w]
            if s_array is None:
                s = np.clip(geom.wire_arc[w], knots[0], knots[-1])
            else:
                s = np.clip(np.asarray(s_array[w], dtype=np.float64), knots[0], knots[-1])
            c = np.zeros(len(knots) - d - 1, dtype=np.complex128)
            for j, _k, _jn, _e, mg in basis.kept[w]:
                c[j] = coeffs[mg]
            out.append(T.basis_values(knots, d, s) @ c if s.size else np.zeros(0, dtype=np.complex128))
        sp = self._enrichment_specs_now()
        if sp and s_array is not None:
            # the enrichment shapes vanish at the knots, so only arcs between
            # knots carry them (bspline.py:4649-4683)
            s_eval = [np.clip(np.asarray(s_array[w], dtype=np.float64), basis.knots[w][0], basis.knots[w][-1])
                      for w in range(len(self.wires_polylines))]
            out = EN.add_between_knots(out, coeffs, sp, geom, s_eval,
                                       EN.shape_polynomial(self.enrichment_variant, d), basis.n)
        return out

    def current_slopes(self, coeffs, s_array=None):
        """Per-wire dI/ds, the solved current's exact arc-length derivative
        (``bspline.py:4523-4584``), at the mesh knots or at the given arc
        positions per wire, clipped into each wire's knot range like
        ``currents_at_knots``.  The derivative of a degree-d B-spline sum is
        the degree-(d-1) sum on the inner knots with coefficients
        d (c_{j+1} - c_j) / (t_{j+d+1} - t_{j+1}); at degree 1 it is
        piecewise constant and a knot takes its right-hand span.  Refused
        under singular enrichment, whose shapes' slope diverges at the
        junction knot (the reference's refusal and text)."""
        if self.use_singular_enrichment:
            raise NotImplementedError(
                "current_slopes does not serve use_singular_enrichment=True: the enrichment shape's slope is "
                "singular at the junction knot, so dropping it would be a silent error rather than an "
                "approximation")
        coeffs = np.asarray(coeffs)
        geom, basis = self._geometry(), self._basis()
        d = self.degree
        out = []
        for w in range(len(self.wires_polylines)):
            knots = basis.knots[w]
            if s_array is None:
                s = np.clip(geom.wire_arc[w], knots[0], knots[-1])
            else:
                s = np.clip(np.asarray(s_array[w], dtype=np.float64), knots[0], knots[-1])
            c = np.zeros(len(knots) - d - 1, dtype=np.complex128)
            for j, _k, _jn, _e, mg in basis.kept[w]:
                c[j] = coeffs[mg]
            if s.size == 0:
                out.append(np.zeros(0, dtype=np.complex128))
                continue
            nb = c.size
            dt = knots[d + 1 : nb + d] - knots[1:nb]
            cd = np.where(dt > 0, d * (c[1:] - c[:-1]) / np.where(dt > 0, dt, 1.0), 0.0)
            out.append(T.basis_values(knots[1:-1], d - 1, s) @ cd)
        return out

    def element_currents(self, coeffs, subdiv: int = 1):
        """(mid, moment, nodes, delta) per mesh element
        (reference ``_element_currents.py:33-120``)."""
        subdiv = int(subdiv)
        if subdiv < 1:
            raise ValueError(f"subdiv must be >= 1, got {subdiv}")
        coeffs = np.asarray(coeffs)
        if coeffs.ndim != 1:
            raise ValueError(
                "element_currents takes ONE solution vector; got coeffs with "
                f"shape {coeffs.shape}. For a multi-port solution pass a single "
                "column, e.g. compute_port_solution().coeffs[:, j]."
            )
        fine, arcs = [], []
        for pl, npe in zip(self.wires_polylines, self.n_per_edge_per_wire):
            parts = []
            for i, n_e in enumerate(npe):
                seg = np.linspace(pl[i], pl[i + 1], n_e * subdiv + 1)
                parts.append(seg if i == 0 else seg[1:])
            knots = np.vstack(parts)
            fine.append(knots)
            step = np.linalg.norm(knots[1:] - knots[:-1], axis=1)
            arcs.append(np.concatenate([[0.0], np.cumsum(step)]))
        currents = self.currents_at_knots(coeffs, None if subdiv == 1 else arcs)
        mids, moments, nodes, deltas = [], [], [], []
        for knots, cur in zip(fine, currents):
            cur = np.asarray(cur)
            element = 0.5 * (cur[1:] + cur[:-1])
            mids.append(0.5 * (knots[1:] + knots[:-1]))
            moments.append(element[:, None] * (knots[1:] - knots[:-1]))
            nodes.append(knots)
            zero = np.zeros(1, dtype=np.complex128)
            deltas.append(np.concatenate([zero, element]) - np.concatenate([element, zero]))
        return (np.concatenate(mids), np.concatenate(moments), np.concatenate(nodes), np.concatenate(deltas))
