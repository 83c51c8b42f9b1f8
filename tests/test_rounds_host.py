"""The round-based propagation (the persistent method's phase kernels),
simulated on the host with the same phase bodies and the same partial state
loads: every track must end bit-identical to the one-shot propagation loop
(propagate_track), whatever the round count, step budget and yield rule.  State a phase does not load is filled with
a poison byte, so a segment that reads a field its phase does not load shows
up as a mismatch."""
import ctypes as C

import numpy as np
import pytest

from detray_b200 import abi, fields, tracks

T = 0.000299792458


def _field_args(fmap):
    if fmap is None:
        return (0, (C.c_double * 3)(0.0, 0.0, 2.0 * T), None, None, None,
                None, None)
    lo = (C.c_double * 3)(*fmap["lo"])
    hi = (C.c_double * 3)(*fmap["hi"])
    nn = (C.c_uint32 * 3)(*fmap["n"])
    vals = np.ascontiguousarray(fmap["values"], dtype=np.float32)
    return (1, (C.c_double * 3)(0.0, 0.0, 0.0), lo, hi, nn,
            vals.ctypes.data_as(C.c_void_p), vals)


def _run(core_host, oracle, det, trk, cfg, fmap, prec, rounds=None,
         budget=16, yield_min=8):
    n = trk.shape[1]
    res, r = oracle.alloc_results(n, cfg.max_records)
    trk = np.ascontiguousarray(trk)
    ptrs = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    kind, b, lo, hi, nn, vp, _keep = _field_args(fmap)
    if rounds is None:
        rc = core_host.core_host_propagate(
            prec, C.byref(det.desc), kind, b, lo, hi, nn, vp, C.byref(cfg),
            ptrs, C.c_uint64(n), C.byref(r))
        stats = None
    else:
        stats = np.zeros(3 * (rounds + 1), np.uint32)
        rc = core_host.core_host_propagate_rounds(
            prec, C.byref(det.desc), kind, b, lo, hi, nn, vp, C.byref(cfg),
            ptrs, C.c_uint64(n), C.byref(r), rounds, budget, yield_min,
            stats.ctypes.data_as(C.c_void_p))
    assert rc == 0, core_host.core_host_last_error()
    return res, stats


def _assert_identical(a, b):
    for key, x in a.items():
        if not isinstance(x, np.ndarray):
            continue
        y = b[key]
        if key == "path_length":
            # the one-shot harness writes the fp64 accumulator, the phases
            # the result type (as the device does)
            x, y = x.astype(np.float32), y.astype(np.float32)
        if x.dtype.kind == "f":
            assert np.array_equal(x, y, equal_nan=True), key
        else:
            assert np.array_equal(x, y), key


def _case(oracle, kind):
    if kind == "telescope_volume_material":
        return (oracle.build_telescope(volume_material="iron"),
                tracks.telescope_tracks(400, seed=8),
                abi.make_config(max_records=16, use_eloss_gradient=1), None)
    if kind == "telescope":
        return (oracle.build_telescope(), tracks.telescope_tracks(400, seed=3),
                abi.make_config(max_records=16), None)
    if kind == "toy_map":
        return (oracle.build_toy(),
                tracks.toy_tracks(800, seed=5, pt_range=(0.1, 100.0)),
                abi.make_config(max_records=32, search_window=(3, 3),
                                estimate_scattering_noise=0),
                fields.solenoid_map())
    if kind == "toy_maps":
        return (oracle.build_toy(use_material_maps=True),
                tracks.toy_tracks(600, seed=6),
                abi.make_config(max_records=32, search_window=(3, 3)), None)
    if kind == "wire":
        return (oracle.build_wire_chamber(square_cells=True),
                tracks.toy_tracks(300, seed=13, pt_range=(0.1, 100.0),
                                  eta_range=(-1.0, 1.0),
                                  vertex_sigma=(0, 0, 0)),
                abi.make_config(max_records=64, search_window=(3, 3),
                                estimate_scattering_noise=0), None)
    return (oracle.build_toy(), tracks.toy_tracks(800, seed=4),
            abi.make_config(max_records=32, search_window=(3, 3)), None)


@pytest.mark.parametrize("kind", ["telescope", "toy", "toy_map", "toy_maps",
                                  "wire", "telescope_volume_material"])
@pytest.mark.parametrize("prec", [4, 8])
def test_rounds_equal_one_shot_loop(core_host, oracle, kind, prec):
    det, trk, cfg, fmap = _case(oracle, kind)
    ref, _ = _run(core_host, oracle, det, trk, cfg, fmap, prec)
    # (rounds, step budget, yield lanes)
    for params in [(300, 16, 8), (300, 4, 30), (7, 3, 16), (40, 1000, 1)]:
        got, stats = _run(core_host, oracle, det, trk, cfg, fmap, prec,
                          *params)
        _assert_identical(ref, got)


def test_rounds_queue_statistics(core_host, oracle):
    """The toy detector's tracks finish within a few dozen rounds (the
    surface actors run inside the step phase, so no track ever waits in the
    surface queue)."""
    det, trk, cfg, fmap = _case(oracle, "toy")
    _, stats = _run(core_host, oracle, det, trk, cfg, fmap, 4, 200, 16, 8)
    q = stats.reshape(-1, 3)
    assert q[:, 1].sum() == 0
    live = np.nonzero(q.sum(axis=1))[0]
    assert 10 < live.max() < 120
    assert q[-1].sum() == 0  # nothing left for the tail
