"""Frozen algorithmic work constants of the propagation path.

FP32 operations per counted device event, counted by hand from the device
code (an FMA counts as 2, add/sub/mul/div/compare-free arithmetic as 1;
transcendental and square-root SFU operations are NOT counted).  Multiplied
with the per-track event counters the kernels write (n_trials, n_steps,
n_intersections, n_transports, n_material), they give the algorithmic FLOPs
of a propagation, from which the roofline fraction is computed.

  F_TRIAL      one RKN4 trial (rk_stepper.hpp:355-430): two stage positions
               (2 x 12), three trial directions (3 x 6), four Lorentz forces
               q/p (t x B) (3 x 12 + first stage outside the loop), error
               vector and norm (~20), step scaling (~6)           = 110
  F_STEP       accepted step: track advance (rk_stepper.hpp:593-629, ~50)
               plus the transport-Jacobian update with covariance transport
               (rk_stepper.hpp:632-956): dk/dqop (4 crosses + 3 scaled
               crosses ~80), dk/dt (4 column-wise crosses 108, 3 block
               additions 54, 4 scalings 36), dF/dt, dG/dt (108), D*J on the
               25 non-trivial entries (~150)                         = 590
  F_ISECT      one ray-surface intersection incl. the mask check: plane
               (dot products 16, division, point 6, point_to_local 18, mask
               ~6, tolerance ~4) ~50; portal cylinder ~30; counted as  50
  F_TRANSPORT  covariance transport to a surface: full bound->bound Jacobian
               (~350), J C J^T on the 4x5 non-trivial block (~340),
               free->bound (~40), noise-free bookkeeping             = 750
  F_MATERIAL   Bethe-Bloch, Landau sigma, Highland, q/p and covariance
               update (~100 without the SFU logs/sqrts)              = 100
"""
from __future__ import annotations

import numpy as np

F_TRIAL = 110
F_STEP = 590
F_ISECT = 50
F_TRANSPORT = 750
F_MATERIAL = 100


def algorithmic_flops(n_trials, n_steps, n_isect, n_transport, n_material) -> float:
    s = lambda a: float(np.asarray(a, dtype=np.float64).sum())  # noqa: E731
    return (F_TRIAL * s(n_trials) + F_STEP * s(n_steps) + F_ISECT * s(n_isect)
            + F_TRANSPORT * s(n_transport) + F_MATERIAL * s(n_material))


def nominal_fp32_tflops(n_sm: int, sm_mhz: float) -> float:
    """FP32 peak: 128 FP32 lanes per SM, one FMA (2 flops) per lane per clock."""
    return n_sm * 128 * 2 * sm_mhz * 1e6 / 1e12
