"""Seeded synthetic track samples for the benchmark configurations.

The reference generates tracks with std::mt19937_64 on the host
(tests/include/detray/test/common/event_generator/random_track_generator.hpp:43-216,
random_numbers.hpp:22-89).  Here numpy's PCG64 generators, seeded explicitly,
produce the same kinds of samples; every consumer (the device propagator and
the reference oracle) reads the same host arrays, so the generator itself
never enters a parity comparison.

All samples are returned as a (8, n) float64 array holding detray's free
vector rows [x, y, z, t, tx, ty, tz, q/p] (track_parametrization.hpp:49-63),
with detray's units (mm, GeV; q in units of e).
"""
from __future__ import annotations

import numpy as np

DEFAULT_SEED = 5489  # std::mt19937_64 default seed used by the reference


def _assemble(pos, dirs, p, q):
    n = p.shape[0]
    out = np.zeros((8, n), dtype=np.float64)
    out[0:3] = pos
    out[3] = 0.0
    norm = np.sqrt((dirs ** 2).sum(axis=0))
    out[4:7] = dirs / norm
    out[7] = q / p
    return out


def telescope_tracks(n: int, seed: int = DEFAULT_SEED, pt: float = 10.0,
                     cone_deg: float = 10.0) -> np.ndarray:
    """Muons from the origin with directions uniform within a cone of
    ``cone_deg`` around +x, transverse momentum (w.r.t. z) ``pt`` GeV and a
    random charge sign."""
    rng = np.random.default_rng(seed)
    cos_max = np.cos(np.deg2rad(cone_deg))
    cos_a = rng.uniform(cos_max, 1.0, n)
    sin_a = np.sqrt(np.maximum(0.0, 1.0 - cos_a ** 2))
    az = rng.uniform(-np.pi, np.pi, n)
    dirs = np.stack([cos_a, sin_a * np.cos(az), sin_a * np.sin(az)])
    perp = np.sqrt(dirs[0] ** 2 + dirs[1] ** 2)
    p = pt / perp
    q = np.where(rng.uniform(0.0, 1.0, n) < 0.5, -1.0, 1.0)
    pos = np.zeros((3, n))
    return _assemble(pos, dirs, p, q)


def toy_tracks(n: int, seed: int = DEFAULT_SEED, pt_range=(1.0, 100.0),
               eta_range=(-4.0, 4.0), vertex_sigma=(0.1, 0.1, 50.0),
               pt_log_uniform: bool = True) -> np.ndarray:
    """Muons from a Gaussian vertex spread, eta uniform in ``eta_range``,
    phi uniform, pT log-uniform (or uniform) in ``pt_range`` GeV, random
    charge sign."""
    rng = np.random.default_rng(seed)
    pos = np.stack([rng.normal(0.0, vertex_sigma[0], n),
                    rng.normal(0.0, vertex_sigma[1], n),
                    rng.normal(0.0, vertex_sigma[2], n)])
    eta = rng.uniform(eta_range[0], eta_range[1], n)
    phi = rng.uniform(-np.pi, np.pi, n)
    if pt_log_uniform:
        pt = np.exp(rng.uniform(np.log(pt_range[0]), np.log(pt_range[1]), n))
    else:
        pt = rng.uniform(pt_range[0], pt_range[1], n)
    theta = 2.0 * np.arctan(np.exp(-eta))
    dirs = np.stack([np.cos(phi) * np.sin(theta), np.sin(phi) * np.sin(theta),
                     np.cos(theta)])
    p = pt / np.sin(theta)
    q = np.where(rng.uniform(0.0, 1.0, n) < 0.5, -1.0, 1.0)
    return _assemble(pos, dirs, p, q)
