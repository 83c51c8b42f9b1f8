"""Reverse-mode derivatives of the propagation (C ABI dprop_propagate_adjoint
and dprop_backward) and their PyTorch autograd binding.

    rec = propagate_differentiable(cfg, det, field, tracks, alignment)
    loss = ((rec[0:2] - targets) ** 2 * weights).sum()
    loss.backward()      # tracks.grad: dL/d(x, y, z, t, tx, ty, tz, q/p)
                         # alignment.grad: dL/d(dt, w) per surface

``rec`` is the (6, max_records, n) tensor of recorded bound parameters
(loc0, loc1, phi, theta, q/p, t) of transported records (zero elsewhere;
``rec_mask`` says which).  ``alignment`` is an (n_surfaces, 6) float64
tensor of surface corrections (dt_x, dt_y, dt_z, w_x, w_y, w_z) at which the
derivative is taken; the propagation runs on the geometry the Detector was
created with, so it must be zero (the derivative at the nominal placement;
``alignment.apply_alignment`` builds a moved geometry for a new Detector).

There is no CPU fallback: everything runs in the sm_100a library.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import abi
from .propagator import (Detector, DeviceResults, Field, PropagationError,
                         _check, alloc_device_results, load_library,
                         make_launch, tracks_struct)


@dataclass
class AdjointRecord:
    """Results and tape of one adjoint-mode propagation."""
    results: DeviceResults
    tape_rec: object    # torch float32 [27, max_records, n]
    tape_init: object   # torch float32 [35, n]
    tape: abi.Tape
    tracks: object      # the (8, n) float32 input tensor
    max_records: int


def _check_tracks(tracks):
    import torch
    if not (hasattr(tracks, "is_cuda") and tracks.is_cuda):
        raise PropagationError("adjoint propagation needs a CUDA tensor")
    if tracks.dtype != torch.float32 or tracks.dim() != 2 or tracks.shape[0] != 8:
        raise PropagationError("tracks must be a (8, n) float32 tensor")


def propagate_adjoint(cfg: abi.Config, det: Detector, field: Field, tracks,
                      launch: abi.Launch | None = None,
                      stream=None) -> AdjointRecord:
    """Adjoint-mode propagation of a (8, n) float32 CUDA tensor."""
    import torch
    _check_tracks(tracks)
    tracks = tracks.detach().contiguous()
    n = tracks.shape[1]
    cap = cfg.max_records
    res = alloc_device_results(n, cap, tracks.device)
    tape_rec = torch.empty((abi.TAPE_RECORD_FLOATS, cap, n),
                           dtype=torch.float32, device=tracks.device)
    tape_init = torch.empty((abi.TAPE_TRACK_FLOATS, n), dtype=torch.float32,
                            device=tracks.device)
    tape = abi.Tape()
    tape.rec = tape_rec.data_ptr()
    tape.init = tape_init.data_ptr()
    if stream is None:
        stream = torch.cuda.current_stream(tracks.device)
    ts = tracks_struct(tracks)
    lc = launch if launch is not None else make_launch(sort_tracks=1)
    _check(load_library().dprop_propagate_adjoint(
        C.byref(cfg), C.byref(lc), det.handle, field.handle, C.byref(ts),
        C.byref(res.struct), C.byref(tape), n, C.c_void_p(stream.cuda_stream)))
    return AdjointRecord(res, tape_rec, tape_init, tape, tracks, cap)


def backward(cfg: abi.Config, det: Detector, rec: AdjointRecord, grad_bound,
             with_alignment: bool = True, stream=None):
    """Reverse sweep for dL/d(rec_bound) = ``grad_bound`` (6, max_records, n)
    float32 CUDA tensor.  Returns (grad_free (8, n) float32, grad_align
    (n_surfaces, 6) float64 or None)."""
    import torch
    n = rec.tracks.shape[1]
    dev = rec.tracks.device
    gb = grad_bound.detach().to(device=dev, dtype=torch.float32).contiguous()
    if tuple(gb.shape) != (6, rec.max_records, n):
        raise PropagationError(
            f"grad_bound must have shape (6, {rec.max_records}, {n})")
    grad_free = torch.empty((8, n), dtype=torch.float32, device=dev)
    grad_align = (torch.zeros((det.n_surfaces, 6), dtype=torch.float64,
                              device=dev) if with_alignment else None)
    g = abi.Gradients()
    for i in range(6):
        g.grad_bound[i] = gb[i].data_ptr()
    for i in range(8):
        g.grad_free[i] = grad_free[i].data_ptr()
    g.grad_align = grad_align.data_ptr() if grad_align is not None else None
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    ts = tracks_struct(rec.tracks)
    _check(load_library().dprop_backward(
        C.byref(cfg), det.handle, C.byref(ts), C.byref(rec.results.struct),
        C.byref(rec.tape), C.byref(g), n, C.c_void_p(stream.cuda_stream)))
    return grad_free, grad_align


def rec_mask(rec: AdjointRecord):
    """(max_records, n) bool: slots holding transported bound parameters."""
    import torch
    t = rec.results.tensors
    cap = rec.max_records
    slot = torch.arange(cap, device=rec.tracks.device)[:, None]
    stored = slot < t["n_records"].clamp(max=cap)[None, :]
    return stored & ((t["rec_flags"] & 1) != 0)


def _make_function():
    import torch

    class Propagation(torch.autograd.Function):
        """Differentiable propagation: tracks (8, n) and alignment
        (n_surfaces, 6) -> recorded bound parameters (6, max_records, n)."""

        @staticmethod
        def forward(ctx, tracks, alignment, cfg, det, field, launch):
            if alignment is not None and bool((alignment != 0).any()):
                raise PropagationError(
                    "alignment must be zero: the derivative is taken at the "
                    "Detector's placements (build a moved Detector instead)")
            rec = propagate_adjoint(cfg, det, field, tracks, launch)
            mask = rec_mask(rec)
            out = torch.where(mask[None], rec.results.tensors["rec_bound"],
                              torch.zeros((), device=tracks.device))
            ctx.rec = rec
            ctx.cfg = cfg
            ctx.det = det
            ctx.want_align = alignment is not None
            ctx.mark_non_differentiable(mask)
            return out, mask

        @staticmethod
        def backward(ctx, grad_out, _grad_mask):
            grad_free, grad_align = backward(
                ctx.cfg, ctx.det, ctx.rec, grad_out,
                with_alignment=ctx.want_align and ctx.needs_input_grad[1])
            return grad_free, grad_align, None, None, None, None

    return Propagation


_FUNCTION = None


def propagate_differentiable(cfg: abi.Config, det: Detector, field: Field,
                             tracks, alignment=None,
                             launch: abi.Launch | None = None):
    """Differentiable propagation (see the module docstring).  Returns
    (rec_bound (6, max_records, n), rec_mask (max_records, n))."""
    global _FUNCTION
    if _FUNCTION is None:
        _FUNCTION = _make_function()
    return _FUNCTION.apply(tracks, alignment, cfg, det, field, launch)
