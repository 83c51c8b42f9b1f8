"""Shared parity checks between a propagation result and the oracle.

Both results use the dprop_results layout (slot-major records).  The checks:
  * per-track status and the sequence of recorded surface barcodes equal,
    except for a bounded number of tracks (``max_seq_mismatch_frac``) whose
    fp32 path grazes a mask boundary and so legitimately crosses a different
    surface (and may then end differently);
  * on tracks with equal sequences, bound parameters and covariance at every
    transported surface within abs + rel tolerances.
"""
from __future__ import annotations

import numpy as np

BOUND_NAMES = ["loc0", "loc1", "phi", "theta", "qop", "time"]


def sequences_equal(a: dict, b: dict) -> np.ndarray:
    n = a["status"].shape[0]
    cap = min(a["rec_barcode"].shape[0], b["rec_barcode"].shape[0])
    na = a["n_records"].astype(np.int64)
    nb = b["n_records"].astype(np.int64)
    ok = na == nb
    slots = np.arange(cap)[:, None]
    valid = slots < np.minimum(na, cap)[None, :]
    ba = a["rec_barcode"][:cap].astype(np.uint64)
    bb = b["rec_barcode"][:cap].astype(np.uint64)
    diff = (ba != bb) & valid
    ok &= ~diff.any(axis=0)
    return ok


def compare(ref: dict, got: dict, *, max_seq_mismatch_frac: float,
            tol_abs: dict, tol_rel: float, cov_rel: float,
            cov_abs_floor: float = 1e-12) -> dict:
    """Returns a summary; raises AssertionError on violation."""
    n = ref["status"].shape[0]
    status_ok = ref["status"] == got["status"]
    seq_ok = sequences_equal(ref, got)
    n_bad_seq = int((~seq_ok).sum())
    assert n_bad_seq <= max_seq_mismatch_frac * n + 1, (
        f"{n_bad_seq} of {n} tracks cross a different surface sequence")
    n_bad_status = int((~status_ok).sum())
    assert n_bad_status <= max_seq_mismatch_frac * n + 1, (
        f"{n_bad_status} of {n} tracks end with a different status")
    good = np.where(seq_ok & status_ok)[0]
    cap = min(ref["rec_barcode"].shape[0], got["rec_barcode"].shape[0])
    nrec = np.minimum(ref["n_records"][good].astype(np.int64), cap)
    mask = (np.arange(cap)[:, None] < nrec[None, :]) & \
        ((ref["rec_flags"][:cap, good] & 1) > 0)
    worst = {}
    for i, name in enumerate(BOUND_NAMES):
        x = ref["rec_bound"][i][:cap, good][mask].astype(np.float64)
        y = got["rec_bound"][i][:cap, good][mask].astype(np.float64)
        err = np.abs(x - y)
        lim = tol_abs[name] + tol_rel * np.abs(x)
        bad = err > lim
        worst[name] = float(err.max()) if err.size else 0.0
        assert not bad.any(), (
            f"{name}: {int(bad.sum())} values out of tolerance, worst "
            f"{err.max():.3e}")
    if "rec_cov" in got and "rec_cov" in ref:
        # covariance: |dC_ij| / sqrt(C_ii C_jj) (correlation scale)
        pairs = [(i, j) for i in range(6) for j in range(i, 6)]
        diag = {i: pairs.index((i, i)) for i in range(6)}
        dref = {i: np.abs(ref["rec_cov"][diag[i]][:cap, good][mask]
                          .astype(np.float64)) for i in range(6)}
        for k, (i, j) in enumerate(pairs):
            x = ref["rec_cov"][k][:cap, good][mask].astype(np.float64)
            y = got["rec_cov"][k][:cap, good][mask].astype(np.float64)
            scale = np.maximum(np.sqrt(dref[i] * dref[j]), cov_abs_floor)
            rel = np.abs(x - y) / scale
            worst[f"cov{i}{j}"] = float(rel.max()) if rel.size else 0.0
            assert not (rel > cov_rel).any(), (
                f"cov[{i}{j}]: {int((rel > cov_rel).sum())} values out of "
                f"tolerance, worst {rel.max():.3e}")
    return {"n": n, "seq_mismatch": n_bad_seq,
            "status_mismatch": int((~status_ok).sum()), "worst": worst}
