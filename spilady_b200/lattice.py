"""Seeded synthetic initial states for bcc Fe (positions, momenta, spins).

The lattice follows the reference's bcc100 builder (bcc100.cpp:33-90): two
atoms per conventional cell at (0,0,0) and (a/2,a/2,a/2), replicated with x
fastest, then y, then z, the whole lattice shifted by a/4 on every axis and
wrapped into the box.  Spins follow initial_spin.cpp:42-52 (moment m along -z,
s = m / -g, so s points along +z with |s| = m0/g), then each is tilted by a
Gaussian polar angle with a uniform azimuth.  Momenta are Maxwell-Boltzmann
draws with the net momentum removed (the reference's initial_momentum.cpp
uses rand() plus a rescale instead; only the distribution is kept).

Units are the reference's internal ones (spilady.h:53-62): Angstrom, eV,
seconds; momenta in eV s / Angstrom so that p^2/m is in eV with the mass in
eV/(Angstrom/s)^2.
"""
from __future__ import annotations

import numpy as np

SPEED_OF_LIGHT = 299792458e0
BOLTZ = 8.617343e-5
UTOEV = 931.494028e6 / SPEED_OF_LIGHT / SPEED_OF_LIGHT
LENGTH_SCALE = 1e-10
HBAR = 6.58211899e-16
EL_G = 2.0023193043622e0

A_FE = 2.8665


def default_params(ncell, a=A_FE):
    """variables.in keys (variables.in:1-22 and default.h:44-226) for a cubic
    box of ``ncell`` conventional cells per axis."""
    L = ncell * a
    return {
        "box": (L, 0.0, L, 0.0, 0.0, L),   # xx yx yy zx zy zz
        "step": 1e-15,
        "temperature": 300.0,              # K
        "atmass": 55.847,                  # u
        "gamma_L_over_mass": 6e11,         # s^-1
        "gamma_S_HL": 5.88e13,
        "rcut_pot": 4.1001,
        "rcut_mag": 3.7501,
        "rcut_max": 4.1001,
        "min_length_link_cell": 4.11,
        "kappa_e": 80.0,
        "random_seed": 1234,
    }


def atmass_internal(atmass_u):
    return atmass_u * UTOEV * LENGTH_SCALE ** 2


def bcc_positions(ncell, a=A_FE):
    n = ncell
    k = np.arange(n, dtype=np.float64)
    z, y, x = np.meshgrid(k, k, k, indexing="ij")
    base = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1) * a
    r = np.empty((base.shape[0] * 2, 3))
    r[0::2] = base
    r[1::2] = base + a / 2.0
    r += a / 4.0
    L = n * a
    return np.mod(r, L)


def initial_state(ncell, *, seed=1, temperature=300.0, tilt=0.05,
                  mag_mom=2.2, pos_sigma=0.0, a=A_FE, atmass_u=55.847):
    """Return (params, r, p, s) for an ncell^3 bcc Fe box."""
    rng = np.random.default_rng(seed)
    params = default_params(ncell, a)
    r = bcc_positions(ncell, a)
    n = r.shape[0]
    if pos_sigma > 0:
        L = ncell * a
        r = np.mod(r + rng.normal(0.0, pos_sigma, size=r.shape), L)
    m = atmass_internal(atmass_u)
    p = rng.normal(0.0, np.sqrt(m * BOLTZ * temperature), size=(n, 3))
    p -= p.mean(axis=0)
    s0 = mag_mom / EL_G
    theta = rng.normal(0.0, tilt, size=n)
    phi = rng.uniform(0.0, 2 * np.pi, size=n)
    s = np.stack([s0 * np.sin(theta) * np.cos(phi),
                  s0 * np.sin(theta) * np.sin(phi),
                  s0 * np.cos(theta)], axis=1)
    return params, r, p, s


def hot_spot_te(ncell_te, box_len, center=None, peak=3000.0, background=300.0,
                sigma=20.0):
    """Gaussian electron-temperature hot spot on an ncell_te^3 mesh (K).

    Node (ix, iy, iz) sits at the centre of its mesh cell; ``sigma`` is in
    Angstrom (2 nm = 20 A); distances use the minimum image."""
    n = ncell_te
    h = box_len / n
    c = np.asarray(center if center is not None else (box_len / 2,) * 3)
    k = (np.arange(n) + 0.5) * h
    z, y, x = np.meshgrid(k, k, k, indexing="ij")
    d = np.stack([x - c[0], y - c[1], z - c[2]], axis=-1)
    d -= box_len * np.round(d / box_len)
    r2 = (d ** 2).sum(-1)
    te = background + (peak - background) * np.exp(-r2 / (2 * sigma ** 2))
    return te.ravel()   # index ix + iy*n + iz*n*n
