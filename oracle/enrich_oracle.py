"""CPU oracle for singular basis enrichment at wire junctions.

TEST INFRASTRUCTURE ONLY.  Only ``tests/`` (and, through them, nothing in
the product) may import this module, and only as the checker.

Restates the reference's enrichment of ``BSplineSolver``
(``use_singular_enrichment=True``; paths relative to ``src/momwire/``):
one extra basis per wire end at every junction of at least
``enrichment_min_k`` wire ends, with the shape u log u (u the normalised
distance from the junction along the adjacent segment) -- or, for the
"stable" variant, u log u minus its L2 projection onto the degree-d bubble
polynomials -- and the augmented Galerkin system
[[Z, Z_pe], [Z_ep, Z_ee]] (``bspline.py:3048-3693``, ``4121-4179``).
Written vectorised over the quadrature grid, not as the reference's loops.
"""

from __future__ import annotations

import numpy as np

from oracle import bspline_oracle as O


def projection_coeffs(d):
    """Monomial coefficients of the L2 projection of t log t onto the
    polynomials of degree <= d on [0, 1] vanishing at 0 and 1
    (``bspline.py:233-300``).  Bubbles b_i = t^(i+1) - t^(i+2), i < d - 1;
    <b_i, b_j> and <t log t, b_i> in closed form
    (int_0^1 t^n dt = 1/(n+1), int_0^1 t^n log t dt = -1/(n+1)^2)."""
    c = np.zeros(d + 1)
    nb = d - 1
    if nb <= 0:
        return c
    G = np.zeros((nb, nb))
    m = np.zeros(nb)
    for i in range(nb):
        for j in range(nb):
            s = i + j
            G[i, j] = 1.0 / (s + 3) - 2.0 / (s + 4) + 1.0 / (s + 5)
        m[i] = -1.0 / (i + 3) ** 2 + 1.0 / (i + 4) ** 2
    a = np.linalg.solve(G, m)
    for i in range(nb):
        c[i + 1] += a[i]
        c[i + 2] -= a[i]
    return c


def specs(spec, geom, min_k=3, active=None):
    """(junction, wire, end, segment, origin) per enrichment basis
    (``bspline.py:3048-3076``): origin 0 when the junction sits at the
    segment's left end (a wire start), 1 at its right end."""
    out = []
    for j, g in enumerate(spec.junctions):
        if len(g) < min_k or (active is not None and j not in active):
            continue
        for w, end in g:
            info = geom["wires"][w]
            if end == "start":
                out.append((j, w, end, info["first"], 0))
            else:
                out.append((j, w, end, info["first"] + info["n"] - 1, 1))
    return out


def _enrich_nodes(geom, sp, t, w, proj):
    """Per enrichment basis: quadrature points (E, q, 3), weight * value and
    weight * arc derivative (E, q)."""
    d = len(proj) - 1
    dproj = proj[1:] * np.arange(1, d + 1)
    pts, wv, wd = [], [], []
    for (_j, _w, _end, s, origin) in sp:
        h = geom["h"][s]
        u = t if origin == 0 else 1.0 - t
        lu = np.log(np.maximum(u, 1e-300))
        val = u * lu - np.polynomial.polynomial.polyval(u, proj)
        dval = (1.0 if origin == 0 else -1.0) * (lu + 1.0 - np.polynomial.polynomial.polyval(u, dproj)) / h
        pts.append(geom["seg_l"][s] + t[:, None] * (geom["seg_r"][s] - geom["seg_l"][s]))
        wv.append(w * h * val)
        wd.append(w * h * dval)
    return np.array(pts), np.array(wv), np.array(wd)


def _poly_nodes(geom, basis, t, w):
    """Per (basis, wing): points (nb, nw, q, 3), weight * value, weight *
    derivative (nb, nw, q); the wing's segment (nb, nw)."""
    supp, polys = basis.supp_seg, basis.polys
    d = polys.shape[2] - 1
    h = geom["h"][supp]  # (nb, nw)
    u = h[..., None] * t  # (nb, nw, q)
    P = u[..., None] ** np.arange(d + 1)  # (nb, nw, q, d+1)
    val = np.einsum("mwqp,mwp->mwq", P, polys)
    dP = np.zeros_like(P)
    dP[..., 1:] = u[..., None] ** np.arange(d) * np.arange(1, d + 1)
    dval = np.einsum("mwqp,mwp->mwq", dP, polys)
    sl, sr = geom["seg_l"][supp], geom["seg_r"][supp]
    pts = sl[:, :, None, :] + t[None, None, :, None] * (sr - sl)[:, :, None, :]
    wq = w * h[..., None]
    return pts, wq * val, wq * dval


def _green(X, Y, a2, k):
    """exp(-j k R) / (4 pi R), R = sqrt(|X - Y|^2 + a^2), X (..., 3) vs Y."""
    diff = X[..., :, None, :] - Y[..., None, :, :]
    R = np.sqrt(np.sum(diff * diff, axis=-1) + a2)
    return np.exp(-1j * k * R) * (O.INV4PI / R)


def _mix(wA, IA, wP, IP, omega):
    """j w mu wA I_A + wP I_P / (j w eps)."""
    return 1j * omega * O.MU0 * wA * IA + wP * IP / (1j * omega * O.EPS0)


def _tangent_weights(t_obs, t_src, spec, geom_c_obs, geom_c_src, omega, image):
    """(w_A, w_Phi) for observer / source segment arrays: the tangent dot in
    free space, the image tables of each ground model otherwise
    (``bspline.py:1575-1650``)."""
    if not image:
        return np.einsum("...i,...i->...", t_obs, t_src) + 0j, np.ones(np.broadcast_shapes(t_obs.shape[:-1],
                                                                                             t_src.shape[:-1]))
    tm = t_src * np.array([1.0, 1.0, -1.0])
    td = np.einsum("...i,...i->...", t_obs, tm)
    if spec.ground_eps is None:
        return td + 0j, np.ones_like(td) + 0j
    et = O.eps_tilde(spec.ground_eps, omega)
    if spec.ground_model == "sommerfeld":
        c2 = (et - 1.0) / (et + 1.0)
        return c2 * td, np.full(td.shape, c2)
    c_o, c_s = np.broadcast_arrays(geom_c_obs, geom_c_src)
    dx = c_o[..., 0] - c_s[..., 0]
    dy = c_o[..., 1] - c_s[..., 1]
    dz = c_o[..., 2] + c_s[..., 2] - 2.0 * spec.ground_z
    hyp = np.hypot(dx, dy)
    rmag = np.maximum(np.sqrt(dx * dx + dy * dy + dz * dz), 1e-30)
    cth = dz / rmag
    safe = hyp > 1e-30
    inv = 1.0 / np.where(safe, hyp, 1.0)
    px = np.where(safe, -dy * inv, 1.0)
    py = np.where(safe, dx * inv, 0.0)
    to, ts = np.broadcast_arrays(t_obs, tm)
    P = (to[..., 0] * px + to[..., 1] * py) * (ts[..., 0] * px + ts[..., 1] * py)
    root = np.sqrt(et - (1.0 - cth * cth) + 0j)
    rv = (et * cth - root) / (et * cth + root)
    rh = (cth - root) / (cth + root)
    wA = rv * (td - P) - rh * P
    mode = spec.ground_phi_mode
    if mode == "rho_v":
        wP = rv
    elif mode == "image":
        wP = np.full(wA.shape, (et - 1.0) / (et + 1.0))
    elif mode == "blend":
        wP = 0.5 * (rv + (et - 1.0) / (et + 1.0))
    else:
        r = np.sqrt(et)
        wP = np.full(wA.shape, (r - 1.0) / (r + 1.0))
    return wA, wP


def blocks(spec, geom, basis, sp, variant="raw", n_qp_sing=32, somm_grid=None):
    """(Z_pe, Z_ep, Z_ee) of the augmented system, the ground's reaction
    subtracted (``bspline.py:3114-3306`` free space, ``3308-3521`` image,
    ``1919-2033`` Sommerfeld remainder)."""
    d = spec.degree
    nb = basis.supp_seg.shape[0]
    E = len(sp)
    Zpe = np.zeros((nb, E), np.complex128)
    Zep = np.zeros((E, nb), np.complex128)
    Zee = np.zeros((E, E), np.complex128)
    if E == 0:
        return Zpe, Zep, Zee
    k, om = spec.k, spec.omega
    a2 = float(spec.radius[0]) ** 2
    t, w = O.gl01(n_qp_sing)
    proj = projection_coeffs(d) if variant == "stable" else np.zeros(d + 1)
    pe, ve, de = _enrich_nodes(geom, sp, t, w, proj)
    seg_e = np.array([s[3] for s in sp])
    tan, cen = geom["tangents"], 0.5 * (geom["seg_l"] + geom["seg_r"])
    pp, vp, dp = _poly_nodes(geom, basis, t, w)
    supp = basis.supp_seg
    live = np.any(basis.polys != 0.0, axis=2)  # (nb, nw)
    gz = spec.ground_z
    passes = [False] + ([True] if gz is not None else [])
    for image in passes:
        sign = -1.0 if image else 1.0
        mir = (lambda x: O.mirror_pts(x, gz)) if image else (lambda x: x)
        # Z_ee[e, f]: observer e, source f
        G = _green(pe[:, None], mir(pe)[None, :], a2, k)  # (E, E, q, q)
        IA = np.einsum("eq,eqfr,fr->ef", ve, G.transpose(0, 2, 1, 3), ve)
        IP = np.einsum("eq,eqfr,fr->ef", de, G.transpose(0, 2, 1, 3), de)
        wA, wP = _tangent_weights(tan[seg_e][:, None], tan[seg_e][None, :], spec, cen[seg_e][:, None],
                                  cen[seg_e][None, :], om, image)
        Zee += sign * _mix(wA, IA, wP, IP, om)
        # Z_pe[m, e] (observer m's wings, source e) and Z_ep[e, m]
        G1 = _green(pp[:, :, None], mir(pe)[None, None], a2, k)  # (nb, nw, E, q, q)
        IA1 = np.einsum("mwq,mweqr,er->mwe", vp, G1, ve)
        IP1 = np.einsum("mwq,mweqr,er->mwe", dp, G1, de)
        wA1, wP1 = _tangent_weights(tan[supp][:, :, None], tan[seg_e][None, None], spec, cen[supp][:, :, None],
                                    cen[seg_e][None, None], om, image)
        Zpe += sign * np.einsum("mwe,mw->me", _mix(wA1, IA1, wP1, IP1, om), live)
        G2 = _green(pe[:, None, None], mir(pp)[None], a2, k)  # (E, nb, nw, q, q)
        IA2 = np.einsum("eq,emwqr,mwr->emw", ve, G2, vp)
        IP2 = np.einsum("eq,emwqr,mwr->emw", de, G2, dp)
        wA2, wP2 = _tangent_weights(tan[seg_e][:, None, None], tan[supp][None], spec, cen[seg_e][:, None, None],
                                    cen[supp][None], om, image)
        Zep += sign * np.einsum("emw,mw->em", _mix(wA2, IA2, wP2, IP2, om), live)
    if gz is not None and spec.ground_eps is not None and spec.ground_model == "sommerfeld":
        from oracle import sommerfeld_oracle as so

        q = spec.n_qp_sommerfeld
        tq, wg = O.gl01(q)
        h = geom["h"]
        nodes = geom["seg_l"][:, None, :] + tq[None, :, None] * (geom["seg_r"] - geom["seg_l"])[:, None, :]
        W = (wg[None, :] * h[:, None])[None] * (h[:, None] * tq[None, :])[None] ** np.arange(d + 1)[:, None, None]
        obs_p = nodes.reshape(-1, 3)
        t_p = np.repeat(tan, q, axis=0)
        obs_e = pe.reshape(-1, 3)
        t_e = np.repeat(tan[seg_e], n_qp_sing, axis=0)
        n_seg = geom["seg_l"].shape[0]
        Fee = so.field_proj(obs_e, t_e, obs_e, t_e, gz, k, somm_grid).reshape(E, n_qp_sing, E, n_qp_sing)
        Zee -= np.einsum("eq,eqfr,fr->ef", ve, Fee, ve)
        Fpe = so.field_proj(obs_p, t_p, obs_e, t_e, gz, k, somm_grid).reshape(n_seg, q, E, n_qp_sing)
        Jpe = np.einsum("piq,iqer,er->pie", W, Fpe, ve)  # (d+1, n_seg, E)
        Fep = so.field_proj(obs_e, t_e, obs_p, t_p, gz, k, somm_grid).reshape(E, n_qp_sing, n_seg, q)
        Jep = np.einsum("eq,eqir,Pir->eiP", ve, Fep, W)  # (E, n_seg, d+1)
        for a in range(supp.shape[1]):
            Zpe -= np.einsum("mp,pme->me", basis.polys[:, a, :], Jpe[:, supp[:, a], :])
            Zep -= np.einsum("emP,mP->em", Jep[:, supp[:, a], :], basis.polys[:, a, :])
    return Zpe, Zep, Zee


def tap_ratios(spec, geom, basis, coeffs, min_k=3):
    """min |I| / max |I| over the wire ends of each junction, from the
    polynomial coefficients of an unenriched solve (``bspline.py:3078-3112``);
    None for junctions below min_k."""
    cur = O.currents_at_knots(spec, geom, basis, coeffs)
    out = []
    for g in spec.junctions:
        if len(g) < min_k:
            out.append(None)
            continue
        mags = [abs(cur[w][0 if end == "start" else -1]) for w, end in g]
        m = max(mags)
        out.append(0.0 if m == 0.0 else min(mags) / m)
    return out


def port_solution(spec, variant="raw", min_k=3, n_qp_sing=32, tikhonov_lambda=1e-3, threshold=0.3,
                  somm_master_values=None):
    """The enriched ``compute_port_solution`` (``bspline.py:4121-4179``):
    returns (Y, coeffs with the enrichment block last, specs used)."""
    geom = O.build_geometry(spec)
    basis = O.build_basis(spec, geom)
    grid = None
    if spec.ground_z is not None and spec.ground_eps is not None and spec.ground_model == "sommerfeld":
        grid = O.sommerfeld_grid(spec, geom, somm_master_values)
    Z = O.compute_Z(spec, geom, basis, somm_master_values)
    B, kcl = O.port_columns(spec, geom, basis)
    active = None
    if variant == "auto":
        X1 = O.solve_ports(Z, B, kcl)
        act = set()
        for j in range(B.shape[1]):
            for i, r in enumerate(tap_ratios(spec, geom, basis, X1[:, j], min_k)):
                if r is not None and r > threshold:
                    act.add(i)
        active = sorted(act)
        if not active:
            return B.T @ X1, X1, []
    sp = specs(spec, geom, min_k, active)
    if not sp:
        X = O.solve_ports(Z, B, kcl)
        return B.T @ X, X, sp
    Zpe, Zep, Zee = blocks(spec, geom, basis, sp, "stable" if variant == "stable" else "raw", n_qp_sing, grid)
    n, E = Z.shape[0], len(sp)
    Za = np.zeros((n + E, n + E), np.complex128)
    Za[:n, :n], Za[:n, n:], Za[n:, :n], Za[n:, n:] = Z, Zpe, Zep, Zee
    if variant == "tikhonov":
        Za[n:, n:] += tikhonov_lambda * float(np.mean(np.abs(np.diag(Zee)))) * np.eye(E)
    Ba = np.zeros((n + E, B.shape[1]), np.complex128)
    Ba[:n] = B
    ka = np.zeros((kcl.shape[0], n + E))
    ka[:, :n] = kcl
    X = O.solve_ports(Za, Ba, ka)
    return B.T @ X[:n], X, sp
