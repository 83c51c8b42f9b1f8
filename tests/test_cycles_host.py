"""Exact stepping cycles (core/propagate.cuh, cycle_search / skip_cycles).

In single precision a low-pT looper can end up in a cycle of a few steps
around a surface it grazes without crossing: each linearised intersection
puts the surface a um or two ahead, the step lands past the turning point
where it lies behind, the track steps back, and the state repeats bit for
bit.  The reference's progress check (propagator.hpp:350-373) passes on
every forward step, so the reference steps the cycle until its path-limit
aborter ends it; its own single-precision build does this on 46 of the 2 M
tracks below, with up to 4.2 M steps for one track.  The core skips the
whole cycles that fit below the path limit and steps the rest; it looks
for cycles only among the states after steps shorter than 1 mm, so cycles
of longer steps (which reach the path limit within a few thousand steps)
are stepped out as in the reference.

Checked here on the host build of the core in single precision, wire
chamber in the solenoid map: against the same build with the skip compiled
out (DPROP_NO_CYCLE_SKIP, every cycle stepped out as in the reference) the
results are bit-identical - status, records, final free parameters, path -
on tracks that cycle and on tracks that do not, and only the step counts
drop.  The tracks are taken from toy_tracks(2 M, seed 20241253, pT 0.1-100
GeV), where this build cycles on 499 of them."""
import ctypes as C

import numpy as np
import pytest

CYCLING = [2694, 112936, 240413, 259424, 417020, 458732, 493033,
           529462, 550560, 630524, 874366, 907295, 938196, 940859, 972325,
           1053854, 1152190, 1258104, 1408405, 1449842, 1547633, 1560741,
           1568187, 1569094, 1686976, 1695669, 1762997, 1771067, 1977017,
           1978546]
# um-step cycles: 117 298, 169 971 and 394 105 trials when stepped out
LONG_CYCLES = [514217, 869041, 1935033]


def _propagate(lib, oracle, desc, cfg, fmap, trk):
    n = trk.shape[1]
    res, r = oracle.alloc_results(n, cfg.max_records)
    trk = np.ascontiguousarray(trk)
    ptrs = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    lo = (C.c_double * 3)(*fmap["lo"])
    hi = (C.c_double * 3)(*fmap["hi"])
    nn = (C.c_uint32 * 3)(*fmap["n"])
    vals = np.ascontiguousarray(fmap["values"], dtype=np.float32)
    rc = lib.core_host_propagate(
        4, C.byref(desc), 1, None, lo, hi, nn,
        vals.ctypes.data_as(C.POINTER(C.c_float)), C.byref(cfg), ptrs,
        C.c_uint64(n), C.byref(r))
    assert rc == 0, lib.core_host_last_error()
    return res


@pytest.fixture(scope="module")
def wire_case():
    from detray_b200 import abi, fields, geometry, tracks
    all_trk = tracks.toy_tracks(2_000_000, seed=20241253,
                                pt_range=(0.1, 100.0))
    trk = np.concatenate([all_trk[:, CYCLING], all_trk[:, LONG_CYCLES],
                          all_trk[:, :3000]], axis=1)
    cfg = abi.make_config(max_records=48, search_window=(3, 3),
                          estimate_scattering_noise=0)
    cfg.max_iterations = 1_000_000
    desc = geometry.Descriptor(geometry.load_geometry(
        "wire_chamber_10l_cells"))
    return cfg, desc, fields.solenoid_map(), trk


def test_cycle_skip_is_exact(core_host, core_host_stepped, oracle,
                             wire_case):
    from detray_b200 import abi
    cfg, desc, fmap, trk = wire_case
    got = _propagate(core_host, oracle, desc.desc, cfg, fmap, trk)
    ref = _propagate(core_host_stepped, oracle, desc.desc, cfg, fmap, trk)
    for k in ("status", "n_records", "rec_barcode", "rec_bound", "rec_cov",
              "final_free", "path_length"):
        assert np.array_equal(got[k], ref[k], equal_nan=True), k
    n_cyc = len(CYCLING) + len(LONG_CYCLES)
    # the cycles end at the path limit in both builds; the um-step ones in
    # a few hundred steps instead of 10^5
    assert np.all(got["status"][:n_cyc] == abi.TRK_PATH_LIMIT)
    assert np.all(got["n_trials"][:n_cyc] <= ref["n_trials"][:n_cyc])
    long = slice(len(CYCLING), n_cyc)
    assert np.all(ref["n_trials"][long] > 100_000)
    assert np.all(got["n_trials"][long] < 1_000)
    # the other tracks take the same steps, but for the odd one that cycles
    # as well (~1 in 4 000)
    fewer = got["n_trials"][n_cyc:] != ref["n_trials"][n_cyc:]
    assert fewer.sum() <= 3
    assert np.all(got["n_trials"][n_cyc:][fewer] < ref["n_trials"][n_cyc:][fewer])
    assert np.all(got["status"][n_cyc:][fewer] == abi.TRK_PATH_LIMIT)
