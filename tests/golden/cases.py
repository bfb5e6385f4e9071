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
}

# Cases stored as Y plus a seeded sample of Z entries (full Z would be large).
SAMPLED = {"array4x4", "array16x16"}

BIG_CASES = {
    "array16x16": lambda: dipole_array(16, 16),
}
