"""Multi-GPU sharding of a track batch (one process per GPU).

Tracks are independent and the detector and field are read-only replicas,
so the forward propagation needs no collective: each rank propagates a
contiguous range of the batch and keeps its results.  The ranges are
balanced by an estimate of each track's work rather than by count, because
low-momentum loopers run to the path limit while stiff tracks leave the
detector after a few hundred mm.

The adjoint adds one exchange: the per-surface alignment gradient
(n_surfaces x 6) and the loss are summed over ranks (one all-reduce);
initial-parameter gradients are per track and stay on their rank.
"""
from __future__ import annotations

import numpy as np

from .units import T


def work_estimate(tracks: np.ndarray, b_field: float = 2.0 * T,
                  r_max: float = 1000.0, z_max: float = 3000.0,
                  path_limit: float = 5000.0) -> np.ndarray:
    """Expected path length of each track (8 x n free parameters): a track
    whose helix diameter 2R stays inside r_max loops until the path limit;
    otherwise it leaves through the barrel (r_max) or the end caps (z_max),
    whichever its polar angle reaches first."""
    d = tracks[4:7]
    qop = tracks[7]
    sin_t = np.hypot(d[0], d[1])
    cos_t = np.abs(d[2])
    p = 1.0 / np.maximum(np.abs(qop), 1e-12)
    pt = p * sin_t
    radius = pt / max(b_field, 1e-30)          # helix radius (mm)
    loops = 2.0 * radius < r_max
    to_barrel = np.where(sin_t > 0, r_max / np.maximum(sin_t, 1e-12), np.inf)
    to_caps = np.where(cos_t > 0, z_max / np.maximum(cos_t, 1e-12), np.inf)
    exit_path = np.minimum(to_barrel, to_caps)
    path = np.where(loops, np.minimum(path_limit, to_caps), exit_path)
    return np.minimum(path, path_limit)


def partition(weights: np.ndarray, world: int) -> list[tuple[int, int]]:
    """Contiguous [start, end) ranges, one per rank, with about equal weight
    sums (prefix-sum split); every index is in exactly one range."""
    n = int(len(weights))
    if world < 1:
        raise ValueError("world must be >= 1")
    if n == 0:
        return [(0, 0)] * world
    w = np.maximum(np.asarray(weights, dtype=np.float64), 0.0)
    if not np.isfinite(w).all() or w.sum() <= 0.0:
        w = np.ones(n)
    cum = np.cumsum(w)
    targets = cum[-1] * np.arange(1, world) / world
    cuts = np.searchsorted(cum, targets, side="left") + 1
    cuts = np.clip(cuts, 0, n)
    bounds = [0, *np.maximum.accumulate(cuts).tolist(), n]
    return [(int(bounds[i]), int(bounds[i + 1])) for i in range(world)]


def shard(tracks: np.ndarray, rank: int, world: int, weights=None):
    """This rank's contiguous slice of the batch and its [start, end)."""
    if weights is None:
        weights = work_estimate(tracks)
    lo, hi = partition(weights, world)[rank]
    return tracks[:, lo:hi], (lo, hi)


def allreduce_alignment(grad_align, loss=None, group=None):
    """Sum the alignment gradient (and the loss, if given) over the ranks of
    ``group`` in one all-reduce; returns (grad_align, loss).  A no-op
    outside an initialised process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return grad_align, loss
    flat = grad_align.reshape(-1)
    if loss is not None:
        lt = torch.as_tensor(loss, dtype=flat.dtype, device=flat.device)
        flat = torch.cat([flat, lt.reshape(1)])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    if loss is not None:
        return flat[:-1].reshape(grad_align.shape), flat[-1]
    return flat.reshape(grad_align.shape), None
