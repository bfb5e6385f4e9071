"""Solver configurations shared by the golden generator and the tests.

Each entry maps a case name to a zero-argument function returning the
``BSplineSolver`` keyword arguments.  The same keywords drive the reference
(golden generation), the oracle and ``momwire_b200``.
"""

from __future__ import annotations

import numpy as np

C_LIGHT = 299_792_458.0
HD = 0.962 * 22 / 4  # half-driver of the reference's 22 m default wavelength


def config1():
    """One straight wire, 21 segments, degree 2, 14.1 MHz, centre feed."""
    return dict(
        wires=[[(-5.05, 0.0, 10.0), (5.05, 0.0, 10.0)]],
        nsegs=21,
        degree=2,
        wire_radius=1e-3,
        wavelength=C_LIGHT / 14.1e6,
    )


def dipole_array(nx, ny, nseg=41, f=300e6, seed=0):
    """nx x ny planar array of z-directed half-wave dipoles, 0.5 lambda pitch,
    length 0.48 lambda * (1 + U(-0.01, 0.01)) drawn in row-major order,
    radius 0.5 mm, a 1 V feed at every centre."""
    lam = C_LIGHT / f
    rng = np.random.default_rng(seed)
    wires, feeds = [], []
    for ix in range(nx):
        for iy in range(ny):
            L = 0.48 * lam * (1 + rng.uniform(-0.01, 0.01))
            x, y = ix * 0.5 * lam, iy * 0.5 * lam
            wires.append(np.array([[x, y, -L / 2], [x, y, L / 2]]))
            feeds.append((len(wires) - 1, None, 1.0))
    return dict(wires=wires, nsegs=nseg, degree=2, wire_radius=0.5e-3, wavelength=lam, feeds=feeds)


LAM_SOMM = C_LIGHT / 28.47e6  # 10 m band


def somm_dipole(height_wl, ground_eps, degree, nseg):
    """Horizontal 0.48-wavelength dipole at the given height over a
    Sommerfeld ground, centre-fed."""
    L, z = 0.48 * LAM_SOMM, height_wl * LAM_SOMM
    return dict(wires=[np.array([[0.0, -L / 2, z], [0.0, L / 2, z]])], nsegs=nseg, degree=degree,
                wavelength=LAM_SOMM, wire_radius=5e-4, ground_z=0.0, ground_eps=ground_eps,
                ground_model="sommerfeld")


def somm_ground_plane():
    """Quarter-wave vertical with four sloping quarter-wave radials joined at
    a feed point 0.05 wavelength above a Sommerfeld ground."""
    lam = LAM_SOMM
    base = np.array([0.0, 0.0, 0.05 * lam])
    wires = [np.array([base, base + [0, 0, 0.25 * lam]])]
    for ang in (0.0, 0.5 * np.pi, np.pi, 1.5 * np.pi):
        tip = base + 0.25 * lam * np.array([0.95 * np.cos(ang), 0.95 * np.sin(ang), 0.0]) + [0, 0, -0.04 * lam]
        wires.append(np.array([base, tip]))
    return dict(wires=wires, nsegs=7, degree=2, wavelength=lam, wire_radius=1e-3, ground_z=0.0,
                ground_eps=(5.0, 0.001), ground_model="sommerfeld",
                junctions=[[(0, "start"), (1, "start"), (2, "start"), (3, "start"), (4, "start")]],
                feeds=[(0, 0.05, 1.0)])


def _star():
    return [
        np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 5.0]]),
        np.array([[0.0, 0.0, 5.0], [3.0, 0.0, 8.0]]),
        np.array([[0.0, 0.0, 5.0], [-3.0, 0.0, 8.0]]),
    ]


CASES = {
    "config1": config1,
    "d1_dipole20": lambda: dict(wires=[np.array([[0, 0, -5.29], [0, 0, 5.29]])], nsegs=20, degree=1),
    "d1_yagi": lambda: dict(
        wires=[np.array([[0.0, 0.0, -HD], [0.0, 0.0, HD]]),
               np.array([[-2.2, 0.0, -1.05 * HD], [-2.2, 0.0, 1.05 * HD]])],
        nsegs=20, degree=1),
    "d1_pec": lambda: dict(wires=[np.array([[-HD, 0.0, 7.0], [HD, 0.0, 7.0]])], nsegs=20, degree=1, ground_z=0.0),
    "d2_vdipole": lambda: dict(
        wires=[np.array([[-4.0, 0.0, 2.0], [0.0, 0.0, 0.0], [4.0, 0.0, 2.0]])], nsegs=8, degree=2),
    "d2_pec": lambda: dict(wires=[np.array([[-5.29, 0, 7.0], [5.29, 0, 7.0]])], nsegs=20, degree=2, ground_z=0.0),
    "d2_refl_normal": lambda: dict(
        wires=[np.array([[-5.29, 0, 4.0], [5.29, 0, 4.0]])], nsegs=20, degree=2, ground_z=0.0,
        ground_eps=(13, 0.005)),
    "d2_refl_rhov": lambda: dict(
        wires=[np.array([[-5.29, 0, 4.0], [0.0, 0.0, 5.5], [5.29, 0, 4.0]])], nsegs=10, degree=2, ground_z=0.0,
        ground_eps=(5, 0.02), ground_phi_mode="rho_v"),
    "d2_refl_blend": lambda: dict(
        wires=[np.array([[-5.29, 0, 4.0], [5.29, 0, 4.0]])], nsegs=16, degree=2, ground_z=0.0,
        ground_eps=(20, 0.01), ground_phi_mode="blend"),
    "d2_refl_image": lambda: dict(
        wires=[np.array([[0.0, 0, 1.0], [0.0, 0, 6.0]])], nsegs=12, degree=2, ground_z=0.0,
        ground_eps=10 - 2j, ground_phi_mode="image"),
    "d2_ek": lambda: dict(
        wires=[np.array([[0, 0, -5.29], [0, 0, 5.29]])], nsegs=20, degree=2, extended_kernel=True, wire_radius=0.05),
    "d2_ek_monopole_pec": lambda: dict(
        wires=[np.array([[0, 0, 0.0], [0, 0, 5.0]])], nsegs=12, degree=2, extended_kernel=True, wire_radius=0.03,
        ground_z=0.0, feeds=[(0, 0.3, 1.0)]),
    "d2_junction": lambda: dict(
        wires=_star(), nsegs=6, degree=2, junctions=[[(0, "end"), (1, "start"), (2, "start")]],
        feeds=[(0, 2.5, 1.0)]),
    "d2_junction_port": lambda: dict(
        wires=_star(), nsegs=6, degree=2, junctions=[[(0, "end"), (1, "start"), (2, "start")]],
        feeds=[(0, 2.5, 1.0)], junction_ports=[0]),
    "d2_node_gap": lambda: dict(
        wires=[np.array([[0, 0, -5.0], [0, 0, 0.0]]), np.array([[0, 0, 0.0], [0, 0, 5.0]])], nsegs=10, degree=2,
        junctions=[[(0, "end"), (1, "start")]], feeds=[], node_gaps=[(1, "start", 1.0)]),
    "d2_monopole_contact": lambda: dict(
        wires=[np.array([[0, 0, 0.0], [0, 0, 5.0]])], nsegs=10, degree=2, ground_z=0.0, feeds=[(0, 0.25, 1.0)]),
    "d2_mixed_radius_kink": lambda: dict(
        wires=[np.array([[0, 0, 0.0], [0, 0, 3.0], [2.0, 0, 5.0]]), np.array([[1.0, 1.0, 0.0], [1.0, 1.0, 4.0]])],
        n_per_edge_per_wire=[[7, 5], 9], degree=2, wire_radius=[1e-3, 4e-3], feeds=[(0, 3.0, 1.0), (1, None, 0.5j)]),
    "d2_segment_feed": lambda: dict(
        wires=[np.array([[0, 0, -5.29], [0, 0, 5.29]])], nsegs=21, degree=2, feed_model="segment"),
    "d1_multifeed": lambda: dict(
        wires=[np.array([[0.0, 0.0, -HD], [0.0, 0.0, HD]]), np.array([[3.0, 0.0, -HD], [3.0, 0.0, HD]])],
        nsegs=20, degree=1, feeds=[(0, None, 1.0), (1, None, 1.0 + 0.5j)]),
    "array4x4": lambda: dipole_array(4, 4),
    # Sommerfeld ground (ground_model="sommerfeld"): remainder grid + C2 image
    "d2_somm_dipole": lambda: somm_dipole(0.1, (10.0, 0.002), degree=2, nseg=21),
    "d1_somm_dipole_low": lambda: somm_dipole(0.03, (13.0, 0.005), degree=1, nseg=20),
    "d2_somm_sea": lambda: somm_dipole(0.05, (81.0, 4.0), degree=2, nseg=15),
    "d2_somm_radials": lambda: somm_ground_plane(),
    "d2_somm_contact": lambda: dict(
        wires=[np.array([[0, 0, 0.0], [0, 0, 0.24 * LAM_SOMM]])], nsegs=12, degree=2, wavelength=LAM_SOMM,
        wire_radius=1e-3, ground_z=0.0, ground_eps=(15.0, 0.01), ground_model="sommerfeld", feeds=[(0, 0.2, 1.0)]),
    "d2_somm_far_pair": lambda: dict(
        wires=[np.array([[0, -0.24 * LAM_SOMM, 0.1 * LAM_SOMM], [0, 0.24 * LAM_SOMM, 0.1 * LAM_SOMM]]),
               np.array([[4.5 * LAM_SOMM, -0.24 * LAM_SOMM, 0.1 * LAM_SOMM],
                         [4.5 * LAM_SOMM, 0.24 * LAM_SOMM, 0.1 * LAM_SOMM]])],
        nsegs=11, degree=2, wavelength=LAM_SOMM, wire_radius=1e-3, ground_z=0.0, ground_eps=(10.0, 0.002),
        ground_model="sommerfeld", feeds=[(0, None, 1.0), (1, None, 1.0)]),
}

CASES["d2_somm_plate8"] = lambda: wire_grid_plate(n_cells=8, size=10.0, n_jports=3)

# distributed series wire loading: skin-effect conductor loss and insulation
SIGMA_CU = 5.8e7
CASES["d2_loaded_dipole"] = lambda: dict(
    wires=[np.array([[0.0, 0.0, -10.15 / 2], [0.0, 0.0, 10.15 / 2]])], nsegs=41, degree=2, wavelength=21.264,
    wire_radius=0.16e-3, wire_conductivity=SIGMA_CU, insulation_radius=0.4e-3, insulation_eps_r=3.0)
CASES["d1_loaded_yagi"] = lambda: dict(
    CASES["d1_yagi"](), wire_conductivity=[SIGMA_CU, np.nan], insulation_radius=[1.5e-3, np.nan],
    insulation_eps_r=[2.3, np.nan])
CASES["d2_loaded_junction_pec"] = lambda: dict(
    CASES["d2_junction"](), ground_z=-0.5, wire_conductivity=3.5e7)
CASES["d2_loaded_mixed_radius"] = lambda: dict(
    CASES["d2_mixed_radius_kink"](), wire_conductivity=[SIGMA_CU, 1.0e6])
LOADED = {name for name in CASES if "_loaded_" in name}

# Sommerfeld-ground cases whose fixtures also carry the grid master tables.
SOMMERFELD = {name for name in CASES if "_somm_" in name}

# Cases stored as Y plus a seeded sample of Z entries (full Z would be large).
SAMPLED = {"array4x4", "array16x16", "plate64_somm"}

def wire_grid_plate(n_cells=64, size=10.0, z=2.0, mono_len=10.0, mono_segs=10, n_jports=7, seed=0,
                    ground=(13.0, 5e-3), f=14.1e6):
    """(n_cells+1)^2-node square wire grid (2 segments per cell edge, radius
    1 mm) at height z over a Sommerfeld ground, a vertical monopole from the
    centre node fed at its base segment, and n_jports seeded junction ports
    at grid nodes other than the centre."""
    m = n_cells + 1
    step = size / n_cells
    xy = lambda i, j: (-size / 2 + i * step, -size / 2 + j * step, z)  # noqa: E731
    wires, nodes = [], {}
    for j in range(m):
        for i in range(n_cells):  # x-directed wire (i, j) -> (i + 1, j)
            wires.append(np.array([xy(i, j), xy(i + 1, j)]))
            nodes.setdefault((i, j), []).append((len(wires) - 1, "start"))
            nodes.setdefault((i + 1, j), []).append((len(wires) - 1, "end"))
    for i in range(m):
        for j in range(n_cells):  # y-directed wire (i, j) -> (i, j + 1)
            wires.append(np.array([xy(i, j), xy(i, j + 1)]))
            nodes.setdefault((i, j), []).append((len(wires) - 1, "start"))
            nodes.setdefault((i, j + 1), []).append((len(wires) - 1, "end"))
    c = (n_cells // 2, n_cells // 2)
    cx, cy, _ = xy(*c)
    wires.append(np.array([(cx, cy, z), (cx, cy, z + mono_len)]))
    mono = len(wires) - 1
    nodes[c].append((mono, "start"))
    keys = sorted(nodes)
    junctions = [nodes[k] for k in keys]
    rng = np.random.default_rng(seed)
    cand = [i for i, k in enumerate(keys) if k != c]
    jports = sorted(int(x) for x in rng.choice(cand, size=n_jports, replace=False))
    npe = [2] * (len(wires) - 1) + [mono_segs]
    return dict(wires=wires, n_per_edge_per_wire=npe, degree=2, wire_radius=1e-3, wavelength=C_LIGHT / f,
                junctions=junctions, junction_ports=jports, feeds=[(mono, 0.5 * mono_len / mono_segs, 1.0)],
                ground_z=0.0, ground_eps=ground, ground_model="sommerfeld")


BIG_CASES = {
    "array16x16": lambda: dipole_array(16, 16),
    "plate64_somm": lambda: wire_grid_plate(),
}


# Singular basis enrichment (t log t bases beside K >= enrichment_min_k
# junctions; bspline.py use_singular_enrichment)
def _fan():
    """Fan dipole: two arms of different length leave each feed-side end,
    a dominant-pair K=3 junction at each side of the feed gap."""
    return [
        np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.4]]),
        np.array([[0.0, 0.0, 0.4], [0.0, 5.1, 0.4]]),
        np.array([[0.0, 0.0, 0.4], [0.0, 3.6, 1.2]]),
        np.array([[0.0, 0.0, 0.0], [0.0, -5.1, 0.0]]),
        np.array([[0.0, 0.0, 0.0], [0.0, -3.6, -0.8]]),
    ]


def _radials(z0=1.0):
    base = np.array([0.0, 0.0, z0])
    wires = [np.array([base, base + [0, 0, 5.0]])]
    for ang in (0.0, 0.5 * np.pi, np.pi, 1.5 * np.pi):
        wires.append(np.array([base, base + 4.8 * np.array([np.cos(ang), np.sin(ang), -0.15])]))
    return wires


_RADIAL_JUNCTION = [[(0, "start"), (1, "start"), (2, "start"), (3, "start"), (4, "start")]]
_STAR_JUNCTION = [[(0, "end"), (1, "start"), (2, "start")]]

ENRICH_CASES = {
    "enr_star_raw": lambda: dict(wires=_star(), nsegs=6, degree=2, junctions=_STAR_JUNCTION, feeds=[(0, 2.5, 1.0)],
                                 use_singular_enrichment=True),
    "enr_star_stable": lambda: dict(wires=_star(), nsegs=6, degree=2, junctions=_STAR_JUNCTION,
                                    feeds=[(0, 2.5, 1.0)], use_singular_enrichment=True,
                                    enrichment_variant="stable"),
    "enr_star_tikhonov": lambda: dict(wires=_star(), nsegs=6, degree=2, junctions=_STAR_JUNCTION,
                                      feeds=[(0, 2.5, 1.0)], use_singular_enrichment=True,
                                      enrichment_variant="tikhonov", tikhonov_lambda=0.05),
    "enr_star_auto": lambda: dict(wires=_star(), nsegs=6, degree=2, junctions=_STAR_JUNCTION,
                                  feeds=[(0, 2.5, 1.0)], use_singular_enrichment=True, enrichment_variant="auto"),
    "enr_star_port": lambda: dict(wires=_star(), nsegs=6, degree=2, junctions=_STAR_JUNCTION,
                                  feeds=[(0, 2.5, 1.0)], junction_ports=[0], use_singular_enrichment=True),
    "enr_star_d1": lambda: dict(wires=_star(), nsegs=8, degree=1, junctions=_STAR_JUNCTION, feeds=[(0, 2.5, 1.0)],
                                use_singular_enrichment=True),
    "enr_fan_auto": lambda: dict(wires=_fan(), nsegs=9, degree=2,
                                 junctions=[[(0, "end"), (1, "start"), (2, "start")],
                                            [(0, "start"), (3, "start"), (4, "start")]],
                                 feeds=[(0, 0.2, 1.0)], use_singular_enrichment=True, enrichment_variant="auto"),
    "enr_fan_raw": lambda: dict(wires=_fan(), nsegs=9, degree=2,
                                junctions=[[(0, "end"), (1, "start"), (2, "start")],
                                           [(0, "start"), (3, "start"), (4, "start")]],
                                feeds=[(0, 0.2, 1.0)], use_singular_enrichment=True),
    "enr_node_gap_mink2": lambda: dict(
        wires=[np.array([[0, 0, -5.0], [0, 0, 0.0]]), np.array([[0, 0, 0.0], [0, 0, 5.0]])], nsegs=10, degree=2,
        junctions=[[(0, "end"), (1, "start")]], feeds=[], node_gaps=[(1, "start", 1.0)],
        use_singular_enrichment=True, enrichment_min_k=2),
    "enr_radials_pec": lambda: dict(wires=_radials(), nsegs=7, degree=2, junctions=_RADIAL_JUNCTION,
                                    feeds=[(0, 0.4, 1.0)], ground_z=0.0, use_singular_enrichment=True),
    "enr_radials_refl": lambda: dict(wires=_radials(), nsegs=7, degree=2, junctions=_RADIAL_JUNCTION,
                                     feeds=[(0, 0.4, 1.0)], ground_z=0.0, ground_eps=(13.0, 0.005),
                                     use_singular_enrichment=True, enrichment_variant="stable"),
    "enr_radials_somm": lambda: dict(somm_ground_plane(), use_singular_enrichment=True),
}
