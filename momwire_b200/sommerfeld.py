"""Sommerfeld ground: remainder-surface grids filled and interpolated on the GPU.

The reference composes a Sommerfeld ground as the C2-scaled exact image plus
a smooth remainder field interpolated from four surfaces tabulated on an
(R1, theta) grid (``_sommerfeld.py``; NEC-2 theory manual section IV).  This
module keeps the reference's grid layout, bucketing and two-level cache
(``SommerfeldGrid`` ``_sommerfeld.py:648-813``, ``get_grid`` ``:1081-1116``)
so that a solve interpolates the same lattice the reference does, and does
the work on the device:

* ``mw_somm_surfaces`` fills a wavelength-normalised master (k2 = 2 pi) for
  each (bucketed eps, r1 bucket): one warp per node of the six contour
  integrals;
* a physical-units view of a master is only a scale of its lengths and a
  value factor (``SommerfeldGrid.scaled_to``, ``:878-914``), passed to the
  kernels in the ``mw_somm_grid`` descriptor -- no table is copied;
* ``mw_somm_remainder_q`` interpolates, projects and integrates the
  remainder into Z (``bspline.py:1791-1915``).

Masters stay resident in device memory (a few hundred KB each) in a FIFO
cache of 32 entries per device.
"""

from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import _lib

C_LIGHT = 299_792_458.0  # masters are filled at omega = k2 * C_LIGHT
MU0_GRID = 4e-7 * math.pi
K2_REF = 2.0 * math.pi

# layout constants (_sommerfeld.py:60-138); the three environment overrides
# are the reference's own
R1_CAP_LAMBDA = float(os.environ.get("MOMWIRE_SOMM_R1_CAP_LAMBDA") or "15.0")
R1_NEAR_LAMBDA = float(os.environ.get("MOMWIRE_SOMM_R1_NEAR_LAMBDA") or "4.0")
EPS_IM_BUCKET = float(os.environ.get("MOMWIRE_SOMM_EPS_IM_BUCKET") or "0.01")
DR_FAR_LAMBDA = 0.2
DTH_FAR_DEG = 2.5
N0_CAP = 513
TH_SPLIT_DEG = 30.0
GRID_RTOL = 1e-6  # SommerfeldGrid's default rtol
MASTER_CACHE_MAX = 32


def _torch():
    import torch

    return torch


def layout(eps_t, k2, r1_max):
    """(r1_max, r_break, r_near, r0_fill, regions) of a grid, regions as
    (r0, r1, dr, th0_deg, th1_deg, dth_deg) (``_sommerfeld.py:688-790``)."""
    lam = 2.0 * math.pi / k2
    r1_max = min(max(float(r1_max), 0.35 * lam), R1_CAP_LAMBDA * lam)
    k1 = k2 * np.sqrt(complex(eps_t))
    if k1.imag > 0:
        k1 = np.conj(k1)
    beat = 2.0 * math.pi / max(abs(k1 - k2), 1e-30) if abs(k1) <= 12.0 * k2 else math.inf
    r_near = min(r1_max, R1_NEAR_LAMBDA * lam)
    dth2_target = min(5.0, float(np.degrees(0.07 * lam / r_near)))
    n_th2 = int(np.ceil(TH_SPLIT_DEG / dth2_target)) + 1
    dth2 = TH_SPLIT_DEG / (n_th2 - 1)
    r_break = 0.2 * lam
    layer = 1.0 / max(abs(k1), 1e-300)
    dr0 = min(0.01 * lam, max(layer / 4.0, r_break / (N0_CAP - 1)))
    r0_fill = 0.5 * dr0 if layer < 0.25 * dr0 else 0.0
    sp = TH_SPLIT_DEG
    regions = [
        (0.0, r_break, 0.01 * lam, 0.0, sp, 10.0),
        (0.0, r_break, dr0, sp, 90.0, 10.0),
        (r_break, r_near, min(0.05 * lam, beat / 6.0), 0.0, sp, dth2),
        (r_break, r_near, min(0.1 * lam, beat / 6.0), sp, 90.0, 10.0),
    ]
    if r1_max > r_near * (1.0 + 1e-9):
        dr_far = DR_FAR_LAMBDA * lam
        regions += [(r_near, r1_max, dr_far, 0.0, sp, DTH_FAR_DEG), (r_near, r1_max, dr_far, sp, 90.0, 10.0)]
    return r1_max, r_break, r_near, r0_fill, regions


def r1_bucket_wl(r1_wl):
    """Round a radius in wavelengths up to the next 1.25^n, floor 0.1
    (``_sommerfeld.py:1048-1055``)."""
    x = max(float(r1_wl), 0.1)
    n = math.ceil(math.log(x, 1.25) - 1e-12)
    b = 1.25 ** n
    if b < r1_wl:
        b *= 1.25
    return float(b)


def eps_bucket(eps_t):
    """Quantise Im(eps~) onto the geometric ladder of EPS_IM_BUCKET steps
    (``_sommerfeld.py:1064-1078``); Re is kept exactly."""
    step = 1.0 + EPS_IM_BUCKET
    if step <= 1.0:
        return eps_t
    re, im = eps_t.real, eps_t.imag
    if not (re > 0.0) or im >= 0.0:
        return eps_t
    return complex(re, -(step ** round(math.log(-im, step))))


class MasterGrid:
    """A wavelength-normalised grid (k2 = 2 pi) resident on one device:
    complex128 (nodes, 4) values, node-major per region."""

    def __init__(self, eps_b, r1b_wl, device, stream, tables=None):
        torch = _torch()
        self.eps_t = complex(eps_b)
        self.k2 = K2_REF
        self.omega = K2_REF * C_LIGHT
        self.mu = MU0_GRID
        self.r1_max, self.r_break, self.r_near, self.r0_fill, regs = layout(self.eps_t, K2_REF, r1b_wl)
        self.regions = []
        r1s, ths, off = [], [], 0
        for idx, (r0, r1, dr, th0, th1, dth) in enumerate(regs):
            n_r = max(int(np.ceil((r1 - r0) / dr)) + 1, 4)
            n_th = int(round((th1 - th0) / dth)) + 1
            rn = r0 + dr * np.arange(n_r)
            tn = np.radians(th0 + dth * np.arange(n_th))
            rr, tt = np.meshgrid(rn, tn, indexing="ij")
            if idx == 1 and self.r0_fill > 0.0:
                rr = rr.copy()
                rr[0, :] = self.r0_fill
            r1s.append(rr.ravel())
            ths.append(tt.ravel())
            self.regions.append(dict(r0=r0, dr=dr, th0=math.radians(th0), dth=math.radians(dth), n_r=n_r, n_th=n_th,
                                     offset=off))
            off += n_r * n_th
        self.n_nodes = off
        if tables is not None:
            # given region tables (4, n_r, n_th): upload instead of filling
            flat = [np.asarray(t, dtype=np.complex128).reshape(4, -1).T for t in tables]
            assert [f.shape[0] for f in flat] == [r["n_r"] * r["n_th"] for r in self.regions]
            self.vals = torch.from_numpy(np.ascontiguousarray(np.concatenate(flat))).to(device)
            self.h2d_bytes = self.vals.numel() * 16
            return
        r1 = np.concatenate(r1s)
        th = np.concatenate(ths)
        rho = np.maximum(r1 * np.cos(th), 0.0)
        h = np.maximum(r1 * np.sin(th), 0.0)
        host = np.ascontiguousarray(np.stack([r1, rho, h, th]))
        nodes = torch.from_numpy(host).to(device)
        self.vals = torch.empty((self.n_nodes, 4), dtype=torch.complex128, device=device)
        lib = _lib.load()
        ws = torch.empty(max(int(lib.mw_somm_surfaces_workspace_size()), 8), dtype=torch.uint8, device=device)
        _lib.call("mw_somm_surfaces", self.n_nodes, nodes[0].data_ptr(), nodes[1].data_ptr(), nodes[2].data_ptr(),
                  nodes[3].data_ptr(), self.eps_t.real, self.eps_t.imag, K2_REF, self.omega, self.mu, GRID_RTOL,
                  self.vals.data_ptr(), ws.data_ptr(), stream)
        self._keep = (nodes, ws)  # alive until the stream has consumed them
        self.h2d_bytes = host.nbytes

    def view(self, k2, omega, mu):
        """``mw_somm_grid`` descriptor of this master scaled to (k2, omega,
        mu) (``SommerfeldGrid.scaled_to``)."""
        scale = self.k2 / float(k2)
        factor = (float(omega) * float(mu)) / (self.omega * self.mu)
        g = _lib.SommGrid()
        g.n_region = len(self.regions)
        for i, reg in enumerate(self.regions):
            g.n_r[i], g.n_th[i], g.offset[i] = reg["n_r"], reg["n_th"], reg["offset"]
            g.r0[i], g.dr[i] = reg["r0"] * scale, reg["dr"] * scale
            g.th0[i], g.dth[i] = reg["th0"], reg["dth"]
        g.r1_max = self.r1_max * scale
        g.r_break = self.r_break * scale
        g.th_split = math.radians(TH_SPLIT_DEG)
        g.r_near = self.r_near * scale
        g.value_scale = factor
        g.vals = self.vals.data_ptr()
        return g

    def tables(self):
        """Host copies of the region tables as (4, n_r, n_th) arrays."""
        v = self.vals.cpu().numpy()
        out = []
        for reg in self.regions:
            n = reg["n_r"] * reg["n_th"]
            out.append(np.ascontiguousarray(v[reg["offset"]:reg["offset"] + n].T.reshape(4, reg["n_r"], reg["n_th"])))
        return out


_MASTERS: dict = {}


def master_key(eps_t, k2, r1_max):
    """(bucketed eps~, r1 bucket in wavelengths) of the master that serves a
    grid of radius r1_max at wavenumber k2 (``get_grid``)."""
    lam = 2.0 * math.pi / float(k2)
    return eps_bucket(complex(eps_t)), r1_bucket_wl(min(float(r1_max) / lam, R1_CAP_LAMBDA))


def get_master(eps_t, k2, r1_max, device, stream):
    """The cached master for (eps~, k2, r1_max), filled on first use."""
    eb, r1b = master_key(eps_t, k2, r1_max)
    dev_index = getattr(device, "index", None)
    key = (dev_index, eb, r1b)
    m = _MASTERS.get(key)
    if m is None:
        while len(_MASTERS) >= MASTER_CACHE_MAX:
            _MASTERS.pop(next(iter(_MASTERS)))
        m = MasterGrid(eb, r1b, device, stream)
        _MASTERS[key] = m
    return m


def clear_cache():
    _MASTERS.clear()


def max_image_distance(seg_l_ptr, seg_r_ptr, n_seg, ground_z, device, stream):
    """Grid-sizing radius: the largest endpoint-to-image-point distance
    over the geometry, x1.001 (``_sommerfeld.py:154-205``)."""
    torch = _torch()
    out = torch.zeros(1, dtype=torch.float64, device=device)
    _lib.call("mw_max_image_distance", int(n_seg), seg_l_ptr, seg_r_ptr, float(ground_z), out.data_ptr(), stream)
    return float(out.cpu().item()) * 1.001
