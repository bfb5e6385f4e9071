"""CPU oracle for the Sommerfeld ground of momwire's B-spline solver.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this module, and only as the
checker.  The product package ``momwire_b200`` never imports it.

A numpy/scipy restatement of the reference's Sommerfeld engine
(``src/momwire/_sommerfeld.py``) and of its B-spline Galerkin remainder block
(``src/momwire/bspline.py:1791-1915``):

* the six lambda-integrals of the NEC-2 theory manual (eqs 148-153, kernels
  D1/D2 of eqs 154-155) on the deformed contours of figs 13-14, with the
  reference's contour waypoints, 24-point Gauss-Legendre rule, bisection
  depth and tail-termination rule (``_sommerfeld.py:208-465``);
* the four interpolation surfaces I_rho^V, I_z^V, I_rho^H, I_phi^H
  (eqs 156-159) and their R1 -> 0 limits (eqs 169-172)
  (``_sommerfeld.py:506-584``);
* the (R1, theta) grid with its 4/6-region layout, 4x4 Lagrange
  interpolation, wavelength-normalised masters and the two-level cache keyed
  by the bucketed (eps, r1) (``_sommerfeld.py:648-915``, ``:1038-1116``);
* the projected remainder field (eqs 143-147, ``_sommerfeld.py:940-1035``)
  and the Galerkin block Q (``bspline.py:1791-1915``).

Bessel and Hankel functions come from ``scipy.special`` (the reference's
pure-Python path uses the same); the product evaluates its own.
"""

from __future__ import annotations

import math

import numpy as np
from scipy.special import hankel2, jv

C_LIGHT = 299_792_458.0  # _constants.py (grid masters use this c)
MU0_GRID = 4e-7 * np.pi  # _sommerfeld.py:147
K2_REF = 2.0 * np.pi  # _sommerfeld.py:144 (masters at lambda = 1)

R1_CAP_LAMBDA = 15.0  # _sommerfeld.py:60
R1_NEAR_LAMBDA = 4.0  # _sommerfeld.py:98
DR_FAR_LAMBDA = 0.2  # _sommerfeld.py:101
DTH_FAR_DEG = 2.5  # _sommerfeld.py:102
N0_CAP = 513  # _sommerfeld.py:109
TH_SPLIT_DEG = 30.0  # _sommerfeld.py:113
EPS_IM_BUCKET = 0.01  # _sommerfeld.py:138

GAUSS_N = 24  # _sommerfeld.py:150-151
GX, GW = np.polynomial.legendre.leggauss(GAUSS_N)
ADAPT_DEPTH = 14  # _sommerfeld.py:154

SURF_KEYS = ("IrhoV", "IzV", "IrhoH", "IphiH")


# ---------------------------------------------------------------- integrands
def gamma(lam, k):
    """(lam^2 - k^2)^(1/2) with NEC's vertical cuts (``_sommerfeld.py:208``)."""
    return np.sqrt(-1j * (lam - k)) * np.sqrt(1j * (lam + k))


def kernels_d12(lam, k1, k2):
    """D1, D2 of eqs 154-155 and gamma_2 (``_sommerfeld.py:213-221``)."""
    g1 = gamma(lam, k1)
    g2 = gamma(lam, k2)
    k1s, k2s = k1 * k1, k2 * k2
    d1 = 2.0 / (g1 + g2) - 2.0 * k2s / (g2 * (k1s + k2s))
    d2 = 2.0 / (k1s * g2 + k2s * g1) - 2.0 / (g2 * (k1s + k2s))
    return d1, d2, g2


def integrands(lam, rho, h, k1, k2, form):
    """The six integrands of eqs 148-153 stacked (6, n)
    (``_sommerfeld.py:234-269``); form "J" = Bessel, "H" = Hankel."""
    lam = np.asarray(lam, dtype=np.complex128)
    d1, d2, g2 = kernels_d12(lam, k1, k2)
    e = np.exp(-g2 * h)
    x = lam * rho
    if form == "J":
        small = np.abs(x) < 1e-6
        xs = np.where(small, 1.0, x)
        b0 = np.where(small, 1.0 - 0.25 * x * x, jv(0, xs))
        b1x = np.where(small, 0.5 - x * x / 16.0, jv(1, xs) / xs)
    else:
        b0 = 0.5 * hankel2(0, x)
        b1x = 0.5 * hankel2(1, x) / x
    l2 = lam * lam
    l3 = l2 * lam
    c = d2 * e
    return np.stack([c * (b1x - b0) * l3, c * g2 * g2 * b0 * lam, c * g2 * (b1x * x) * l2,
                     -c * b1x * l3, c * b0 * lam, d1 * e * b0 * lam])


def gl_segment(f, z0, z1):
    """24-point Gauss-Legendre over the straight segment z0 -> z1."""
    mid, half = 0.5 * (z0 + z1), 0.5 * (z1 - z0)
    return f(mid + half * GX) @ (GW * half)


def adaptive(f, z0, z1, rtol, depth=ADAPT_DEPTH, whole=None):
    """Bisection with a tolerance relative to the local magnitude
    (``_sommerfeld.py:280-302``)."""
    if whole is None:
        whole = gl_segment(f, z0, z1)
    mid = 0.5 * (z0 + z1)
    left, right = gl_segment(f, z0, mid), gl_segment(f, mid, z1)
    better = left + right
    err = np.max(np.abs(better - whole))
    if depth <= 0 or err <= rtol * max(np.max(np.abs(better)), 1e-300):
        return better
    return adaptive(f, z0, mid, rtol, depth - 1, left) + adaptive(f, mid, z1, rtol, depth - 1, right)


def tail(f, z0, direction, panel, rtol, ref_scale, panel0=None, max_panels=800):
    """Panel tail toward direction * infinity; stops after two consecutive
    panels below rtol * scale; the first panels ramp geometrically from
    panel0 (``_sommerfeld.py:305-339``)."""
    total = 0.0
    quiet = 0
    z = z0
    step = panel if panel0 is None else min(panel0, panel)
    for _ in range(max_panels):
        z_next = z + step * direction
        contrib = gl_segment(f, z, z_next)
        total = total + contrib
        z = z_next
        step = min(2.0 * step, panel)
        scale = max(np.max(np.abs(total)), ref_scale)
        cmax = np.max(np.abs(contrib))
        if cmax == 0.0 or cmax < rtol * scale:
            quiet += 1
            if quiet >= 2:
                break
        else:
            quiet = 0
    return total


def six_integrals(eps_t, k2, rho, h, rtol=1e-9, form=None):
    """The six integrals at one (rho, h) (``_sommerfeld.py:342-465``):
    Bessel form on the fig-13 contour for rho < 2h, Hankel form on the
    fig-14 contour otherwise."""
    eps_t = complex(eps_t)
    if eps_t == 1.0:
        return np.zeros(6, dtype=np.complex128)
    k2, rho, h = float(k2), float(rho), float(h)
    k1 = k2 * np.sqrt(eps_t)
    if k1.imag > 0:
        k1 = np.conj(k1)
    scale = max(rho, h)
    panel = 0.2 * np.pi / scale
    kmax = max(abs(k1), k2)
    kcap = 1.2 * k2 + 50.0 / scale
    kmax_eff = min(kmax, kcap)
    qtol = min(rtol, 1e-11)
    use_bessel = rho < 2.0 * h if form is None else form == "J"
    if use_bessel:
        def f(lam):
            return integrands(lam, rho, h, k1, k2, "J")

        p = min(1.0 / rho if rho > 0 else np.inf, 1.0 / h)
        brk = p * (1.0 + 1.0j)
        end_adapt = 1.3 * kmax_eff + 3.0 * p + 1.0j * p
        total = adaptive(f, 0.0 + 0.0j, brk, qtol)
        start = brk
        if end_adapt.real > brk.real:
            total = total + adaptive(f, brk, end_adapt, qtol)
            start = end_adapt
        return total + tail(f, start, 1.0 + 0.0j, panel, rtol, np.max(np.abs(total)))

    def f(lam):
        return integrands(lam, rho, h, k1, k2, "H")

    r1 = math.hypot(rho, h)
    dir_right = (h - 1.0j * rho) / r1
    dir_left = (-h - 1.0j * rho) / r1
    a = -0.4j * k2
    b = (0.6 + 0.2j) * k2
    c = (1.02 + 0.2j) * k2
    k1_dead = k1.real * h - k1.imag * rho >= 50.0
    cap_d = kcap if (k1_dead or abs(k1) > 200.0 * k2) else max(kcap, 1.01 * k1.real)
    if 1.01 * k1.real <= cap_d:
        d = 1.01 * k1.real + 0.99j * max(k1.imag, -cap_d)
    else:
        d = cap_d + 0.0j
    if d.real < 1.1 * k2:
        d = 1.1 * k2 + 1.0j * d.imag
    total = adaptive(f, a, b, qtol)
    total = total + adaptive(f, b, c, qtol)
    total = total + adaptive(f, c, d, qtol)
    ref = np.max(np.abs(total))
    p0 = 0.5 * kmax
    total = total + tail(f, d, dir_right, panel, rtol, ref, panel0=p0)
    return total - tail(f, a, dir_left, panel, rtol, ref, panel0=p0)


# ------------------------------------------------------------------ surfaces
def c1_norm(k2, omega, mu):
    """Eq 123 unit-moment normalisation (``_sommerfeld.py:506``)."""
    return -1j * omega * mu / (4.0 * np.pi * k2 * k2)


def limits_r1_zero(eps_t, k2, theta, omega, mu):
    """Eqs 169-172 (``_sommerfeld.py:511-532``)."""
    k1s, k2s = k2 * k2 * complex(eps_t), k2 * k2
    c1 = c1_norm(k2, omega, mu)
    c2 = (k1s - k2s) / (k1s + k2s)
    c3 = k2s * (k1s - k2s) / (k1s + k2s) ** 2
    s, co = np.sin(theta), np.cos(theta)
    near = np.abs(co) < 1e-8
    cs = np.where(near, 1.0, co)
    q1 = np.where(near, 0.0, (1.0 - s) / cs)
    q2 = np.where(near, 0.5, (1.0 - s) / (cs * cs))
    return np.stack([c1 * c3 * k1s * q1, np.full(np.shape(q1), c1 * c3 * k1s, dtype=np.complex128),
                     c1 * k2s * (c2 - c3 + c3 * q2), -c1 * k2s * (c2 - c3 * q2)])


def surfaces_at(eps_t, k2, r1, rho, h, theta, omega, mu, rtol):
    """(4, n) surfaces at nodes given by (R1, rho, h, theta)
    (``_sommerfeld.py:535-584``)."""
    r1 = np.asarray(r1, dtype=float).ravel()
    out = np.zeros((4, r1.size), dtype=np.complex128)
    k1s, k2s = k2 * k2 * complex(eps_t), k2 * k2
    c1 = c1_norm(k2, omega, mu)
    zero = r1 == 0.0
    if np.any(zero):
        out[:, zero] = limits_r1_zero(eps_t, k2, np.asarray(theta, dtype=float).ravel()[zero], omega, mu)
    for i in np.nonzero(~zero)[0]:
        v_rr, v_zz, v_rz, v_r1, v, u = six_integrals(eps_t, k2, rho[i], h[i], rtol)
        ph = c1 * r1[i] * np.exp(1j * k2 * r1[i])
        out[:, i] = [ph * k1s * v_rz, ph * k1s * (v_zz + k2s * v), ph * k2s * (v_rr + u), -ph * k2s * (v_r1 + u)]
    return out


def surfaces_direct(eps_t, k2, R1, theta, rtol=1e-9, omega=None, mu=MU0_GRID):
    """Direct surfaces at (R1, theta) points (``_sommerfeld.py:535``)."""
    omega = k2 * C_LIGHT if omega is None else omega
    R1, theta = np.broadcast_arrays(np.asarray(R1, dtype=float), np.asarray(theta, dtype=float))
    r, t = R1.ravel(), theta.ravel()
    rho = np.maximum(r * np.cos(t), 0.0)
    h = np.maximum(r * np.sin(t), 0.0)
    return surfaces_at(eps_t, k2, r, rho, h, t, omega, mu, rtol).reshape((4,) + R1.shape)


# ---------------------------------------------------------------------- grid
def grid_layout(eps_t, k2, r1_max):
    """Region table of the interpolation grid (``_sommerfeld.py:688-813``):
    returns (r1_max, r_break, r_near, r0_fill, [(r0, r1, dr, th0, th1, dth)])."""
    lam = 2.0 * np.pi / k2
    r1_max = min(max(float(r1_max), 0.35 * lam), R1_CAP_LAMBDA * lam)
    k1 = k2 * np.sqrt(complex(eps_t))
    if k1.imag > 0:
        k1 = np.conj(k1)
    beat = 2.0 * np.pi / max(abs(k1 - k2), 1e-30) if abs(k1) <= 12.0 * k2 else np.inf
    r_near = min(r1_max, R1_NEAR_LAMBDA * lam)
    dth2_target = min(5.0, np.degrees(0.07 * lam / r_near))
    n_th2 = int(np.ceil(TH_SPLIT_DEG / dth2_target)) + 1
    dth2 = TH_SPLIT_DEG / (n_th2 - 1)
    r_break = 0.2 * lam
    layer = 1.0 / max(abs(k1), 1e-300)
    dr0 = min(0.01 * lam, max(layer / 4.0, r_break / (N0_CAP - 1)))
    r0_fill = 0.5 * dr0 if layer < 0.25 * dr0 else 0.0
    sp = TH_SPLIT_DEG
    layout = [
        (0.0, r_break, 0.01 * lam, 0.0, sp, 10.0),
        (0.0, r_break, dr0, sp, 90.0, 10.0),
        (r_break, r_near, min(0.05 * lam, beat / 6.0), 0.0, sp, dth2),
        (r_break, r_near, min(0.1 * lam, beat / 6.0), sp, 90.0, 10.0),
    ]
    if r1_max > r_near * (1.0 + 1e-9):
        dr_far = DR_FAR_LAMBDA * lam
        layout += [(r_near, r1_max, dr_far, 0.0, sp, DTH_FAR_DEG), (r_near, r1_max, dr_far, sp, 90.0, 10.0)]
    return r1_max, r_break, r_near, r0_fill, layout


def grid_nodes(r0, r1, dr, th0, th1, dth):
    """Lattice of one region: (R1 nodes, theta nodes in radians, n_r, n_th)."""
    n_r = max(int(np.ceil((r1 - r0) / dr)) + 1, 4)
    n_th = int(round((th1 - th0) / dth)) + 1
    return r0 + dr * np.arange(n_r), np.radians(th0 + dth * np.arange(n_th)), n_r, n_th


def lagrange4(u):
    """Cubic Lagrange weights for nodes 0..3 at u (``_sommerfeld.py:815``)."""
    u0, u1, u2, u3 = u, u - 1.0, u - 2.0, u - 3.0
    return np.stack([-u1 * u2 * u3 / 6.0, u0 * u2 * u3 / 2.0, -u0 * u1 * u3 / 2.0, u0 * u1 * u2 / 6.0], axis=-1)


class Grid:
    """(R1, theta) interpolation grid of the four surfaces
    (``SommerfeldGrid``, ``_sommerfeld.py:648-915``).  ``values`` may supply
    the region tables (4, n_r, n_th) instead of filling them here."""

    def __init__(self, eps_t, k2, r1_max, rtol=1e-6, omega=None, mu=MU0_GRID, values=None):
        self.eps_t = complex(eps_t)
        self.k2 = float(k2)
        self.omega = self.k2 * C_LIGHT if omega is None else float(omega)
        self.mu = float(mu)
        self.r1_max, self.r_break, self.r_near, self.r0_fill, layout = grid_layout(self.eps_t, self.k2, r1_max)
        self.regions = []
        for idx, (r0, r1, dr, th0, th1, dth) in enumerate(layout):
            rn, tn, n_r, n_th = grid_nodes(r0, r1, dr, th0, th1, dth)
            if values is not None:
                vals = np.asarray(values[idx], dtype=np.complex128)
                assert vals.shape == (4, n_r, n_th), (vals.shape, n_r, n_th)
            else:
                rr, tt = np.meshgrid(rn, tn, indexing="ij")
                if idx == 1 and self.r0_fill > 0.0:
                    rr = rr.copy()
                    rr[0, :] = self.r0_fill
                vals = surfaces_direct(self.eps_t, self.k2, rr, tt, rtol, self.omega, self.mu)
            self.regions.append(dict(r0=r0, dr=dr, n_r=n_r, th0=np.radians(th0), dth=np.radians(dth), n_th=n_th,
                                     vals=vals))

    def node_lists(self):
        """Per region: (rr, tt) node coordinates as filled (R1 = r0_fill on
        region 1's first row when that applies)."""
        out = []
        for idx, reg in enumerate(self.regions):
            rn = reg["r0"] + reg["dr"] * np.arange(reg["n_r"])
            tn = reg["th0"] + reg["dth"] * np.arange(reg["n_th"])
            rr, tt = np.meshgrid(rn, tn, indexing="ij")
            if idx == 1 and self.r0_fill > 0.0:
                rr = rr.copy()
                rr[0, :] = self.r0_fill
            out.append((rr, tt))
        return out

    def eval(self, R1, theta):
        """(4, n) interpolated surfaces (``_sommerfeld.py:831-875``)."""
        r = np.minimum(np.asarray(R1, dtype=float).ravel(), self.r1_max)
        th = np.clip(np.asarray(theta, dtype=float).ravel(), 0.0, 0.5 * np.pi)
        grazing = th <= np.radians(TH_SPLIT_DEG)
        region_of = np.where(r <= self.r_break, np.where(grazing, 0, 1),
                             np.where(r <= self.r_near, np.where(grazing, 2, 3), np.where(grazing, 4, 5)))
        out = np.empty((4, r.size), dtype=np.complex128)
        for idx, reg in enumerate(self.regions):
            sel = np.nonzero(region_of == idx)[0]
            if sel.size == 0:
                continue
            fr = (r[sel] - reg["r0"]) / reg["dr"]
            ft = (th[sel] - reg["th0"]) / reg["dth"]
            i0 = np.clip(np.floor(fr).astype(int) - 1, 0, reg["n_r"] - 4)
            j0 = np.clip(np.floor(ft).astype(int) - 1, 0, reg["n_th"] - 4)
            wr, wt = lagrange4(fr - i0), lagrange4(ft - j0)
            ii = i0[:, None] + np.arange(4)[None, :]
            jj = j0[:, None] + np.arange(4)[None, :]
            block = reg["vals"][:, ii[:, :, None], jj[:, None, :]]
            out[:, sel] = np.einsum("snij,ni,nj->sn", block, wr, wt)
        return out

    def scaled_to(self, k2, omega, mu):
        """Physical-units view of a wavelength-normalised master
        (``_sommerfeld.py:878-914``): lengths x lambda_new/lambda_old,
        values x (omega mu)/(omega_old mu_old)."""
        scale = self.k2 / float(k2)
        factor = (float(omega) * float(mu)) / (self.omega * self.mu)
        g = object.__new__(Grid)
        g.eps_t, g.k2, g.omega, g.mu = self.eps_t, float(k2), float(omega), float(mu)
        g.r1_max, g.r_break, g.r_near = self.r1_max * scale, self.r_break * scale, self.r_near * scale
        g.r0_fill = self.r0_fill * scale
        g.regions = [dict(reg, r0=reg["r0"] * scale, dr=reg["dr"] * scale, vals=reg["vals"] * factor)
                     for reg in self.regions]
        return g


def r1_bucket_wl(r1_wl):
    """Next 1.25^n wavelengths, floor 0.1 (``_sommerfeld.py:1048-1055``)."""
    x = max(float(r1_wl), 0.1)
    n = math.ceil(math.log(x, 1.25) - 1e-12)
    b = 1.25 ** n
    if b < r1_wl:
        b *= 1.25
    return float(b)


def eps_bucket(eps_t):
    """Im(eps) onto the 1% geometric ladder (``_sommerfeld.py:1064-1078``)."""
    step = 1.0 + EPS_IM_BUCKET
    re, im = eps_t.real, eps_t.imag
    if not (re > 0.0) or im >= 0.0:
        return eps_t
    return complex(re, -(step ** round(math.log(-im, step))))


_MASTERS: dict = {}


def get_grid(eps_t, k2, r1_max, omega, mu, master_values=None):
    """Grid for (eps, k2, r1_max, omega, mu) as ``get_grid`` builds it
    (``_sommerfeld.py:1081-1116``): a master at k2 = 2 pi for the bucketed
    (eps, r1) scaled to k2.  ``master_values`` supplies the master's region
    tables (a golden fixture) instead of filling them."""
    k2 = float(k2)
    lam = 2.0 * np.pi / k2
    r1b = r1_bucket_wl(min(float(r1_max) / lam, R1_CAP_LAMBDA))
    eb = eps_bucket(complex(eps_t))
    key = (eb, r1b)
    if master_values is not None:
        master = Grid(eb, K2_REF, r1b, omega=K2_REF * C_LIGHT, mu=MU0_GRID, values=master_values)
    else:
        master = _MASTERS.get(key)
        if master is None:
            master = Grid(eb, K2_REF, r1b, omega=K2_REF * C_LIGHT, mu=MU0_GRID)
            _MASTERS[key] = master
    return master.scaled_to(k2, omega, mu)


def master_key(eps_t, k2, r1_max):
    """(bucketed eps, r1 bucket in wavelengths) of the master a solve uses."""
    lam = 2.0 * np.pi / float(k2)
    return eps_bucket(complex(eps_t)), r1_bucket_wl(min(float(r1_max) / lam, R1_CAP_LAMBDA))


def max_image_distance(seg_l, seg_r, gz):
    """Largest observer-to-image-point distance over endpoint pairs, x1.001
    (``_sommerfeld.py:154-205``)."""
    ex = np.concatenate([seg_l, seg_r])
    dx = ex[:, 0][:, None] - ex[:, 0][None, :]
    dy = ex[:, 1][:, None] - ex[:, 1][None, :]
    hz = (ex[:, 2][:, None] - gz) + (ex[:, 2][None, :] - gz)
    return float(np.sqrt(dx * dx + dy * dy + hz * hz).max()) * 1.001


# ----------------------------------------------------------------- remainder
def field_proj(obs, t_obs, src, t_src, gz, k, grid):
    """t_obs . F(r_obs, r_src) . t_src for every (observer, source) point
    pair (eqs 143-147, ``_sommerfeld.py:940-1035``)."""
    th_src = np.hypot(t_src[:, 0], t_src[:, 1])
    safe_t = th_src > 1e-12
    ux = np.where(safe_t, t_src[:, 0] / np.where(safe_t, th_src, 1.0), 1.0)
    uy = np.where(safe_t, t_src[:, 1] / np.where(safe_t, th_src, 1.0), 0.0)
    tz = t_src[:, 2]
    dx = obs[:, 0][:, None] - src[:, 0][None, :]
    dy = obs[:, 1][:, None] - src[:, 1][None, :]
    rho = np.hypot(dx, dy)
    hh = (obs[:, 2] - gz)[:, None] + (src[:, 2] - gz)[None, :]
    r1 = np.sqrt(rho * rho + hh * hh)
    s = grid.eval(r1, np.arctan2(hh, rho)).reshape((4,) + r1.shape)
    g = np.exp(-1j * k * r1) / r1
    safe_r = rho > 1e-12 * grid.r1_max
    inv = np.where(safe_r, 1.0 / np.where(safe_r, rho, 1.0), 0.0)
    dhx = np.where(safe_r, dx * inv, ux[None, :])
    dhy = np.where(safe_r, dy * inv, uy[None, :])
    cphi = ux[None, :] * dhx + uy[None, :] * dhy
    sphi = ux[None, :] * dhy - uy[None, :] * dhx
    e_rho = g * (tz[None, :] * s[0] + th_src[None, :] * cphi * s[2])
    e_phi = g * th_src[None, :] * sphi * s[3]
    e_z = g * (tz[None, :] * s[1] - th_src[None, :] * cphi * s[0])
    return (t_obs[:, 0][:, None] * (dhx * e_rho - dhy * e_phi) + t_obs[:, 1][:, None] * (dhy * e_rho + dhx * e_phi)
            + t_obs[:, 2][:, None] * e_z)


def remainder_Q(geom, supp_seg, polys, degree, n_qp, gz, k, grid):
    """Galerkin block Q[m, n] = sum f_m f_n t_m . F . t_n over n_qp
    Gauss nodes per segment (``bspline.py:1791-1915``)."""
    seg_l, seg_r, tang, h = geom["seg_l"], geom["seg_r"], geom["tangents"], geom["h"]
    n_seg = seg_l.shape[0]
    xg, wg = np.polynomial.legendre.leggauss(n_qp)
    tq = 0.5 * (xg + 1.0)
    nodes = seg_l[:, None, :] + tq[None, :, None] * (seg_r - seg_l)[:, None, :]
    u = h[:, None] * tq[None, :]
    w = 0.5 * h[:, None] * wg[None, :]
    W = w[None] * u[None] ** np.arange(degree + 1)[:, None, None]  # (d+1, n_seg, q)
    pts = nodes.reshape(-1, 3)
    tt = np.repeat(tang, n_qp, axis=0)
    F = field_proj(pts, tt, pts, tt, gz, k, grid).reshape(n_seg, n_qp, n_seg, n_qp)
    Jc = np.einsum("piq,iqjr,Pjr->pPij", W, F, W)
    nb = polys.shape[0]
    Q = np.zeros((nb, nb), dtype=np.complex128)
    for a in range(degree + 1):
        sm = supp_seg[:, a]
        for b in range(degree + 1):
            sn = supp_seg[:, b]
            Q += np.einsum("mp,pPmn,nP->mn", polys[:, a, :], Jc[:, :, sm[:, None], sn[None, :]], polys[:, b, :])
    return Q
