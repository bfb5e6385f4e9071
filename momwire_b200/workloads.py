"""Seeded synthetic structures for the benchmark workloads.

Every generator returns ``BSplineSolver`` keyword arguments and draws its
randomness from ``numpy.random.default_rng(seed)`` in a fixed order, so a
workload is reproducible from its name and seed alone.
"""

from __future__ import annotations

import numpy as np

C_LIGHT = 299_792_458.0


def dipole_array(nx=16, ny=16, nseg=41, f=300e6, seed=0):
    """nx x ny planar array of z-directed dipoles at 0.5 lambda pitch in x
    and y, z = 0; each 0.48 lambda long with a +-1 % uniform length jitter
    drawn in row-major order; radius 0.5 mm; nseg segments; degree 2; a 1 V
    delta-gap feed at every centre (nx*ny ports)."""
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


def yagi(rng, f0=28e6):
    """One seeded Yagi-Uda: 3-12 parallel z-directed elements spaced along x
    by U(0.10, 0.30) lambda0, lengths U(0.40, 0.55) lambda0, radius
    log-uniform 0.5-10 mm, odd segment counts U{11..101} per element;
    element 1 (after the reflector) is centre-fed with 1 V."""
    lam = C_LIGHT / f0
    n_el = int(rng.integers(3, 13))
    x = 0.0
    wires, npe = [], []
    for e in range(n_el):
        if e:
            x += rng.uniform(0.10, 0.30) * lam
        L = rng.uniform(0.40, 0.55) * lam
        wires.append(np.array([[x, 0.0, -L / 2], [x, 0.0, L / 2]]))
        npe.append(int(2 * rng.integers(5, 51) + 1))
    radius = float(np.exp(rng.uniform(np.log(0.5e-3), np.log(10e-3))))
    return dict(wires=wires, n_per_edge_per_wire=npe, degree=2, wire_radius=radius, wavelength=lam,
                feeds=[(1, None, 1.0)])


def yagi_sweep(n_structures=512, n_freq=64, seed=0):
    """The batched-sweep workload: seeded Yagis, each solved at n_freq
    frequencies uniform over 25.2-30.8 MHz.  Returns (list of kwargs, k)."""
    rng = np.random.default_rng(seed)
    structs = [yagi(rng) for _ in range(n_structures)]
    f = np.linspace(25.2e6, 30.8e6, n_freq)
    eps, mu = 8.8541878188e-12, 1.25663706127e-6
    c = 1.0 / np.sqrt(eps * mu)
    return structs, 2 * np.pi * f / c


def somm_structure(rng):
    """One seeded antenna over a Sommerfeld ground: a horizontal dipole, a
    vertical monopole with 4-16 radials, or an inverted V with a 90-150
    degree apex; lowest point log-uniform 0.02-1 lambda above the ground;
    f U(3, 30) MHz; eps_r U(3, 40); sigma log-uniform 1e-4-1e-1 S/m; 21-201
    segments in total; degree 2; radius 1 mm; 1 V feed."""
    kind = int(rng.integers(0, 3))
    f = rng.uniform(3e6, 30e6)
    lam = C_LIGHT / f
    hgt = float(np.exp(rng.uniform(np.log(0.02), np.log(1.0)))) * lam
    er = rng.uniform(3.0, 40.0)
    sig = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-1))))
    n_total = int(rng.integers(21, 202))
    common = dict(degree=2, wire_radius=1e-3, wavelength=lam, ground_z=0.0, ground_eps=(er, sig),
                  ground_model="sommerfeld")
    if kind == 0:
        L = 0.48 * lam
        n = n_total | 1
        return dict(wires=[np.array([[0.0, -L / 2, hgt], [0.0, L / 2, hgt]])], nsegs=n, **common)
    if kind == 1:
        n_rad = int(rng.integers(4, 17))
        per = max(n_total // (n_rad + 1), 1)
        base = np.array([0.0, 0.0, hgt])
        wires = [np.array([base, base + [0.0, 0.0, 0.25 * lam]])]
        for i in range(n_rad):
            a = 2.0 * np.pi * i / n_rad
            wires.append(np.array([base, base + 0.25 * lam * np.array([np.cos(a), np.sin(a), 0.0])]))
        return dict(wires=wires, nsegs=per, junctions=[[(w, "start") for w in range(n_rad + 1)]],
                    feeds=[(0, 0.5 * 0.25 * lam / per, 1.0)], **common)
    apex = np.radians(rng.uniform(90.0, 150.0))
    leg = 0.25 * lam
    dz, dy = leg * np.cos(apex / 2), leg * np.sin(apex / 2)
    top = np.array([0.0, 0.0, hgt + dz])
    n = max(n_total // 2, 1)
    return dict(wires=[np.array([top - [0.0, dy, dz], top, top + [0.0, dy, -dz]])],
                n_per_edge_per_wire=[[n, n]], **common)


def somm_structures(n_structures=256, seed=0):
    """The Sommerfeld-ground workload: seeded structures of somm_structure."""
    rng = np.random.default_rng(seed)
    return [somm_structure(rng) for _ in range(n_structures)]
