"""Magnetic field maps for the propagation benchmarks.

The inhomogeneous-field configurations use an ideal finite solenoid (a thin
cylindrical current sheet): coil radius R, half-length L, scaled so that the
field at the centre is B0.  It is evaluated analytically in double precision
as a superposition of circular current loops along the coil; the field of
one loop of radius a at (r, z - z') is the classic complete-elliptic-integral
form (e.g. Jackson, Classical Electrodynamics, §5.5):

    k^2 = 4 a r / ((a + r)^2 + dz^2)
    B_z = C / sqrt((a + r)^2 + dz^2) * [K(k) + (a^2 - r^2 - dz^2) /
                                          ((a - r)^2 + dz^2) E(k)]
    B_r = C dz / (r sqrt((a + r)^2 + dz^2)) * [-K(k) + (a^2 + r^2 + dz^2) /
                                          ((a - r)^2 + dz^2) E(k)]

The map is sampled on the regular (r, phi, z) node grid of the device field
(``dprop_field_create_grid``): one phi node (axial symmetry), values
(B_r, B_phi = 0, B_z) in detray's units (1 T = 0.000299792458).
"""
from __future__ import annotations

import numpy as np
from scipy import special

from .units import T


def _loop_field(a, r, dz):
    """(B_r, B_z) of a unit loop of radius a at radial distance r and axial
    offset dz, up to the common factor mu0 I / (2 pi)."""
    r = np.asarray(r, dtype=np.float64)
    dz = np.asarray(dz, dtype=np.float64)
    ap = (a + r) ** 2 + dz ** 2
    am = (a - r) ** 2 + dz ** 2
    m = 4.0 * a * r / ap  # k^2
    m = np.clip(m, 0.0, 1.0 - 1e-15)
    K = special.ellipk(m)
    E = special.ellipe(m)
    sq = np.sqrt(ap)
    bz = (K + (a * a - r * r - dz * dz) / am * E) / sq
    with np.errstate(invalid="ignore", divide="ignore"):
        br = dz / (r * sq) * (-K + (a * a + r * r + dz * dz) / am * E)
    br = np.where(r > 0.0, br, 0.0)
    return br, bz


def solenoid_field(r, z, radius=1200.0, half_length=3000.0, b0=2.0 * T,
                   n_loops=1200):
    """(B_r, B_z) of the finite solenoid at cylindrical points (r, z)."""
    r = np.asarray(r, dtype=np.float64)
    z = np.asarray(z, dtype=np.float64)
    # midpoint rule over the current sheet
    zs = (np.arange(n_loops) + 0.5) / n_loops * 2.0 * half_length - half_length
    br = np.zeros(np.broadcast(r, z).shape)
    bz = np.zeros_like(br)
    for z0 in zs:
        a, b = _loop_field(radius, r, z - z0)
        br += a
        bz += b
    # normalise to b0 at the centre
    _, bz0 = _loop_field(radius, np.array([0.0]), -zs)
    scale = b0 / bz0.sum()
    return br * scale, bz * scale


def solenoid_map(radius=1200.0, half_length=3000.0, b0=2.0 * T,
                 r_max=1500.0, z_max=3500.0, spacing=20.0,
                 n_loops=1200) -> dict:
    """Field map spec for ``propagator.Field.grid`` and the oracle: nodes
    every ``spacing`` mm over r in [0, r_max], |z| <= z_max, one phi node."""
    n_r = int(round(r_max / spacing)) + 1
    n_z = int(round(2.0 * z_max / spacing)) + 1
    rs = np.linspace(0.0, r_max, n_r)
    zs = np.linspace(-z_max, z_max, n_z)
    R, Z = np.meshgrid(rs, zs)  # (n_z, n_r)
    br, bz = solenoid_field(R, Z, radius, half_length, b0, n_loops)
    values = np.zeros((n_z, 1, n_r, 3), dtype=np.float32)
    values[:, 0, :, 0] = br
    values[:, 0, :, 2] = bz
    return {"kind": "grid", "lo": (0.0, -np.pi, -z_max),
            "hi": (r_max, np.pi, z_max), "n": (n_r, 1, n_z),
            "values": values}
