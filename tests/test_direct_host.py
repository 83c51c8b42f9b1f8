"""Direct navigation (core/direct.cuh) on the CPU: the host build of the core
against the reference's propagator with the direct_navigator
(core/include/detray/navigation/direct_navigator.hpp), both fed the
surface sequence the caching navigator collected - the records of a normal
propagation, as the surface_sequencer actor collects them.

Checked as the reference's own test does
(tests/integration_tests/cpu/propagator/propagation_direct_navigator.cpp):
forward along the sequence the same surfaces are reached in the same order
with the same momentum, and backward from the last surface the sequence is
walked in reverse and the start momentum comes back.  In double precision
the core equals the reference operation for operation (parameters to
~1e-12)."""
import ctypes as C

import numpy as np
import pytest

from tests.parity import compare
from tests.test_core_host_parity import TIGHT, T

FIELD = {"kind": "const", "b": (0, 0, 2 * T)}


def core_direct(core_host, oracle, det_desc, cfg, seq, lens, direction,
                trk=None, start_barcode=None, start_bound=None, precision=8):
    n = len(lens)
    res, r = oracle.alloc_results(n, cfg.max_records)
    b = (C.c_double * 3)(0.0, 0.0, 2.0 * T)
    seq = np.ascontiguousarray(seq, dtype=np.uint64)
    lens = np.ascontiguousarray(lens, dtype=np.uint32)
    keep = [seq, lens]
    tp = None
    if trk is not None:
        trk = np.ascontiguousarray(trk, dtype=np.float64)
        keep.append(trk)
        tp = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    sp = None
    sbc = None
    if start_barcode is not None:
        sbc = np.ascontiguousarray(start_barcode, dtype=np.uint64)
        sb = np.ascontiguousarray(start_bound, dtype=np.float64)
        keep += [sbc, sb]
        sp = (C.c_void_p * 6)(*[sb[i].ctypes.data for i in range(6)])
    rc = core_host.core_host_propagate_direct(
        precision, C.byref(det_desc), b, C.byref(cfg), tp, C.c_uint64(n),
        C.c_void_p(seq.ctypes.data) if seq.size else None,
        C.c_void_p(lens.ctypes.data), C.c_uint32(seq.shape[0]),
        C.c_int32(direction),
        C.c_void_p(sbc.ctypes.data) if sbc is not None else None, sp,
        C.byref(r))
    assert rc == 0, core_host.core_host_last_error()
    return res


def last_records(res, lens):
    """Barcode and bound parameters of each track's last record."""
    idx = np.arange(len(lens))
    last = np.maximum(lens.astype(np.int64) - 1, 0)
    return res["rec_barcode"][last, idx], res["rec_bound"][:, last, idx]


def _detector(oracle, kind):
    from detray_b200 import abi, tracks
    if kind == "wire":
        det = oracle.build_wire_chamber(square_cells=True)
        trk = tracks.toy_tracks(300, seed=31, pt_range=(1.0, 20.0),
                                eta_range=(-1.0, 1.0),
                                vertex_sigma=(0, 0, 0))
    else:
        det = oracle.build_toy(use_material_maps=kind == "toy_maps")
        trk = tracks.toy_tracks(400, seed=32, pt_range=(1.0, 20.0))
    cfg = abi.make_config(max_records=64, search_window=(3, 3),
                          estimate_scattering_noise=0)
    return det, cfg, trk


@pytest.mark.parametrize("kind", ["toy", "toy_maps", "wire"])
def test_direct_forward_and_backward_match_reference(core_host, oracle, kind):
    det, cfg, trk = _detector(oracle, kind)
    ref = oracle.propagate(det, FIELD, cfg, trk)
    seq = ref["rec_barcode"]
    lens = np.minimum(ref["n_records"], cfg.max_records)
    assert lens.mean() > 5

    fw_ref = oracle.propagate_direct(det, FIELD, cfg, seq, lens, 1,
                                     tracks=trk)
    fw = core_direct(core_host, oracle, det.desc, cfg, seq, lens, 1, trk=trk)
    s = compare(fw_ref, fw, max_seq_mismatch_frac=0.0, tol_abs=TIGHT,
                tol_rel=1e-7, cov_rel=1e-5)
    assert s["seq_mismatch"] == 0 and s["status_mismatch"] == 0
    # the direct run reaches exactly the collected surfaces, in order
    assert np.all(fw["status"] == 0)
    assert np.array_equal(fw["n_records"], ref["n_records"])
    for t in range(len(lens)):
        assert np.array_equal(fw["rec_barcode"][:lens[t], t],
                              seq[:lens[t], t])
    # same momentum at the last surface as the caching navigator's run
    _, b_ref = last_records(ref, lens)
    _, b_fw = last_records(fw, lens)
    np.testing.assert_allclose(1 / np.abs(b_fw[4]), 1 / np.abs(b_ref[4]),
                               rtol=2e-3)

    sbc, sb = last_records(fw, lens)
    bw_ref = oracle.propagate_direct(det, FIELD, cfg, seq, lens, -1,
                                     start_barcode=sbc, start_bound=sb)
    bw = core_direct(core_host, oracle, det.desc, cfg, seq, lens, -1,
                     start_barcode=sbc, start_bound=sb)
    s = compare(bw_ref, bw, max_seq_mismatch_frac=0.0, tol_abs=TIGHT,
                tol_rel=1e-7, cov_rel=1e-5)
    assert s["seq_mismatch"] == 0 and s["status_mismatch"] == 0
    # walked in reverse; the energy lost forward is regained
    for t in range(len(lens)):
        assert np.array_equal(bw["rec_barcode"][:lens[t], t],
                              seq[:lens[t], t][::-1])
    p0 = 1 / np.abs(trk[7])
    np.testing.assert_allclose(1 / np.abs(bw["final_free"][7]), p0,
                               rtol=2e-3)
    assert np.all(np.abs(bw["final_free"][7]) <= np.abs(fw["final_free"][7])
                  * (1 + 1e-12))


def test_direct_edge_cases(core_host, oracle):
    """Empty sequences end at once without records; a barcode outside the
    detector ends the track as unreachable; lengths above the capacity of
    the sequence array are cut to it."""
    from detray_b200 import abi, tracks
    det = oracle.build_toy()
    cfg = abi.make_config(max_records=16, search_window=(3, 3))
    trk = tracks.toy_tracks(4, seed=33)
    ref = oracle.propagate(det, FIELD, cfg, trk)
    seq = ref["rec_barcode"].copy()
    lens = np.minimum(ref["n_records"], cfg.max_records).astype(np.uint32)
    assert np.all(lens >= 2)
    lens[0] = 0                       # empty
    seq[1, 1] = np.uint64(0x1fffff) << np.uint64(27)  # index beyond the detector
    lens[2] = 1000                    # longer than the array: cut to 16
    got = core_direct(core_host, oracle, det.desc, cfg, seq, lens, 1, trk=trk)
    assert got["status"][0] == abi.TRK_EXITED and got["n_records"][0] == 0
    # the first surface is reached, but the next one cannot be intersected:
    # the navigation aborts inside that update, before the actors run
    assert got["status"][1] == abi.TRK_NO_SURFACE
    assert got["n_records"][1] == 0
    ref_direct = oracle.propagate_direct(det, FIELD, cfg, seq[:, [0, 2, 3]],
                                         lens[[0, 2, 3]], 1,
                                         tracks=trk[:, [0, 2, 3]])
    assert ref_direct["status"][0] == abi.TRK_EXITED
    assert got["status"][2] == ref_direct["status"][1]
    assert got["n_records"][2] == ref_direct["n_records"][1]
    # a bound start on a surface outside the detector
    sbc = np.full(4, np.uint64(0x1fffff) << np.uint64(27), dtype=np.uint64)
    sb = np.zeros((6, 4))
    sb[4] = 0.1
    got = core_direct(core_host, oracle, det.desc, cfg, seq, lens, -1,
                      start_barcode=sbc, start_bound=sb)
    assert np.all(got["status"] == abi.TRK_NO_SURFACE)
