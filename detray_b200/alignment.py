"""Surface alignment on the flat detector tables.

An alignment correction of surface s is a translation ``dt`` and a rotation
vector ``w`` (axis times angle, global axes) about the surface centre:
    x' = c + dt + R(w) (x - c)
so the surface placement (R, c) becomes (R(w) R, c + dt).  This is the
parameterisation the adjoint's alignment gradient (``dL/d(dt, w)`` at
``dt = w = 0``, six values per surface in the order dt_x, dt_y, dt_z, w_x,
w_y, w_z) refers to.  The reference stores each placement and its inverse
(algebra/generic/impl/generic_transform3.hpp); both are rewritten here.
"""
from __future__ import annotations

import numpy as np


def rotation_matrix(w) -> np.ndarray:
    """Rotation by the angle |w| about the axis w (Rodrigues' formula)."""
    w = np.asarray(w, dtype=np.float64)
    a = float(np.linalg.norm(w))
    if a == 0.0:
        return np.eye(3)
    k = w / a
    K = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
    return np.eye(3) + np.sin(a) * K + (1.0 - np.cos(a)) * (K @ K)


def apply_alignment(tables: dict, deltas: dict) -> dict:
    """Copy of ``tables`` with surface placements moved.

    ``deltas`` maps a surface index to its six alignment values
    (dt_x, dt_y, dt_z, w_x, w_y, w_z).  A placement shared with another
    surface or a volume cannot be moved alone and raises ValueError.
    """
    out = {k: np.array(v, copy=True) for k, v in tables.items()}
    surfaces = out["surfaces"]
    trf = out["transforms"]
    if deltas:
        used = np.bincount(surfaces["transform"].astype(np.int64),
                           minlength=len(trf))
        used[out["volumes"]["transform"].astype(np.int64)] += 1
    for s, delta in deltas.items():
        ti = int(surfaces["transform"][s])
        if used[ti] != 1:
            raise ValueError(f"surface {s}: placement {ti} is shared")
        delta = np.asarray(delta, dtype=np.float64)
        R = trf["rot"][ti].reshape(3, 3).T      # column-major -> matrix
        c = np.array(trf["translation"][ti], dtype=np.float64)
        Rn = rotation_matrix(delta[3:]) @ R
        cn = c + delta[:3]
        trf["rot"][ti] = Rn.T.reshape(9)
        trf["translation"][ti] = cn
        inv = Rn.T
        trf["inv_rot"][ti] = inv.T.reshape(9)
        trf["inv_translation"][ti] = -(inv @ cn)
    return out
