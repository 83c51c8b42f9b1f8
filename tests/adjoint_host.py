"""Test helpers: adjoint-mode propagation and the reverse sweep through the
test-only host build of the core (tests/native/core_host.cpp), in double
precision, plus the loss and finite-difference machinery the adjoint tests
share."""
from __future__ import annotations

import ctypes as C

import numpy as np

from detray_b200 import geometry
from oracle import ref_oracle

K_TAPE_REC = 27
K_TAPE_INIT = 35
T = 0.000299792458


def _field_args(field):
    if field is None or field.get("kind", "const") == "const":
        b = field["b"] if field else (0.0, 0.0, 2.0 * T)
        return (0, (C.c_double * 3)(*b), None, None, None, None, None)
    lo = (C.c_double * 3)(*field["lo"])
    hi = (C.c_double * 3)(*field["hi"])
    nn = (C.c_uint32 * 3)(*field["n"])
    vals = np.ascontiguousarray(field["values"], dtype=np.float32)
    return (1, None, lo, hi, nn,
            vals.ctypes.data_as(C.POINTER(C.c_float)), vals)


def forward(core_host, tables, cfg, trk, field=None, adjoint=True):
    """Propagate ``trk`` (8 x n, double) with the host core.  Returns the
    result dict (ref_oracle.alloc_results layout) and, in adjoint mode, the
    tape arrays (rec: [27][cap][n], init: [35][n])."""
    desc = geometry.Descriptor(tables)
    n = trk.shape[1]
    cap = cfg.max_records
    res, r = ref_oracle.alloc_results(n, cap)
    trk = np.ascontiguousarray(trk, dtype=np.float64)
    ptrs = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    kind, b, lo, hi, nn, vals, _keep = _field_args(field)
    if adjoint:
        tape_rec = np.zeros((K_TAPE_REC, cap, n), dtype=np.float64)
        tape_init = np.zeros((K_TAPE_INIT, n), dtype=np.float64)
        rc = core_host.core_host_propagate_adjoint(
            8, C.byref(desc.desc), kind, b, lo, hi, nn, vals, C.byref(cfg),
            ptrs, C.c_uint64(n), C.byref(r),
            tape_rec.ctypes.data_as(C.c_void_p),
            tape_init.ctypes.data_as(C.c_void_p))
        assert rc == 0, core_host.core_host_last_error()
        return res, {"rec": tape_rec, "init": tape_init}
    rc = core_host.core_host_propagate(8, C.byref(desc.desc), kind, b, lo, hi,
                                       nn, vals, C.byref(cfg), ptrs,
                                       C.c_uint64(n), C.byref(r))
    assert rc == 0, core_host.core_host_last_error()
    return res, None


def backward(core_host, tables, cfg, trk, res, tape, grad_bound):
    """Reverse sweep: (grad_free [8][n], grad_align [n_surfaces][6])."""
    desc = geometry.Descriptor(tables)
    n = trk.shape[1]
    trk = np.ascontiguousarray(trk, dtype=np.float64)
    tptr = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    bound = np.ascontiguousarray(res["rec_bound"])
    bptr = (C.c_void_p * 6)(*[bound[i].ctypes.data for i in range(6)])
    gb = np.ascontiguousarray(grad_bound, dtype=np.float64)
    gptr = (C.c_void_p * 6)(*[gb[i].ctypes.data for i in range(6)])
    gfree = np.zeros((8, n), dtype=np.float64)
    fptr = (C.c_void_p * 8)(*[gfree[i].ctypes.data for i in range(8)])
    galign = np.zeros((len(tables["surfaces"]), 6), dtype=np.float64)
    rc = core_host.core_host_backward(
        C.byref(desc.desc), C.c_uint32(cfg.max_records), tptr, C.c_uint64(n),
        res["n_records"].ctypes.data_as(C.c_void_p),
        res["rec_barcode"].ctypes.data_as(C.c_void_p),
        res["rec_flags"].ctypes.data_as(C.c_void_p), bptr,
        tape["rec"].ctypes.data_as(C.c_void_p),
        tape["init"].ctypes.data_as(C.c_void_p), gptr, fptr,
        galign.ctypes.data_as(C.c_void_p))
    assert rc == 0, core_host.core_host_last_error()
    return gfree, galign


def transported_mask(res, cap):
    """[cap][n] bool: record slots that carry bound parameters."""
    n = res["n_records"].shape[0]
    slot = np.arange(cap)[:, None]
    valid = slot < np.minimum(res["n_records"], cap)[None, :]
    return valid & ((res["rec_flags"] & 1) != 0)


def random_weights(res, cap, seed, components=(0, 1, 2, 3, 4)):
    """Random loss weights W [6][cap][n] on the transported records; the
    loss is L = sum(W * rec_bound)."""
    rng = np.random.default_rng(seed)
    n = res["n_records"].shape[0]
    W = np.zeros((6, cap, n))
    mask = transported_mask(res, cap)
    scale = {0: 1.0, 1: 1.0, 2: 100.0, 3: 100.0, 4: 1.0e3}
    for c in components:
        W[c] = rng.normal(0.0, scale.get(c, 1.0), (cap, n)) * mask
    return W


def loss_difference(res_p, res_m, W):
    """Per-track sum W * (b+ - b-), with angle-like components wrapped (the
    records must be the same surfaces in both runs)."""
    d = res_p["rec_bound"] - res_m["rec_bound"]
    for c in (1, 2):  # ring loc1 and phi wrap at +-pi
        d[c] = np.where(d[c] > np.pi, d[c] - 2 * np.pi, d[c])
        d[c] = np.where(d[c] < -np.pi, d[c] + 2 * np.pi, d[c])
    return (W * d).sum(axis=(0, 1))


def same_records(res_a, res_b) -> np.ndarray:
    """Per track: the two runs crossed the same surfaces (stored slots)."""
    na = np.asarray(res_a["n_records"]).astype(np.int64)
    nb = np.asarray(res_b["n_records"]).astype(np.int64)
    bca = np.asarray(res_a["rec_barcode"]).view(np.uint64)
    bcb = np.asarray(res_b["rec_barcode"]).view(np.uint64)
    cap = bca.shape[0]
    stored = np.arange(cap)[:, None] < np.minimum(na, cap)[None, :]
    return (na == nb) & ((bca == bcb) | ~stored).all(axis=0)
