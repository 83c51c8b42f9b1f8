"""Helix truth scan (core/helix.cuh) on the CPU: the host build of the core
against the reference's detector scan with its helix intersectors
(detector_scanner::run<helix_scan>, tests/include/detray/test/validation/
detector_scanner.hpp): same surfaces in the same order for every track, and
in double precision the same path lengths and local positions to ~1e-12
(both run the same Newton-Raphson/bisection iteration)."""
import ctypes as C

import numpy as np
import pytest

from tests.test_core_host_parity import T

B = (0.0, 0.0, 2.0 * T)


def core_scan(core_host, oracle, det_desc, trk, mask_tol, capacity=256,
              b=B):
    n = trk.shape[1]
    res = oracle.alloc_scan(n, capacity)
    trk = np.ascontiguousarray(trk, dtype=np.float64)
    ptrs = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    bb = (C.c_double * 3)(*b)
    rc = core_host.core_host_helix_scan(
        C.byref(det_desc), bb, ptrs, C.c_uint64(n), C.c_double(mask_tol),
        C.c_uint32(capacity),
        *[C.c_void_p(p) for p in oracle.scan_pointers(res)])
    assert rc == 0, core_host.core_host_last_error()
    return res


def assert_scans_match(ref, got, tol):
    from detray_b200 import abi
    assert np.array_equal(ref["status"], got["status"])
    assert np.array_equal(ref["n_hits"], got["n_hits"])
    ok = ref["status"] == abi.SCAN_OK
    for t in np.nonzero(ok)[0]:
        k = ref["n_hits"][t]
        assert np.array_equal(ref["barcode"][:k, t], got["barcode"][:k, t])
        assert np.array_equal(ref["volume_link"][:k, t],
                              got["volume_link"][:k, t])
        for f in ("path", "loc0", "loc1"):
            np.testing.assert_allclose(got[f][:k, t], ref[f][:k, t],
                                       rtol=0, atol=tol)


@pytest.mark.parametrize("kind", ["telescope", "toy", "toy_maps",
                                  "wire_cells", "wire_straws"])
def test_scan_matches_reference(core_host, oracle, kind):
    from detray_b200 import tracks
    if kind == "telescope":
        det = oracle.build_telescope()
        trk = tracks.telescope_tracks(200, seed=51)
    elif kind.startswith("toy"):
        det = oracle.build_toy(use_material_maps=kind == "toy_maps")
        trk = tracks.toy_tracks(60, seed=52, pt_range=(0.5, 50.0))
    else:
        det = oracle.build_wire_chamber(square_cells=kind == "wire_cells")
        trk = tracks.toy_tracks(150, seed=53, pt_range=(0.5, 50.0),
                                eta_range=(-1.0, 1.0))
    ref = oracle.helix_scan(det, B, trk, 1e-3)
    got = core_scan(core_host, oracle, det.desc, trk, 1e-3)
    assert ref["n_hits"].mean() > 5
    assert_scans_match(ref, got, 1e-9)


def test_scan_edge_cases(core_host, oracle):
    """A track that crosses nothing is reported empty; more hits than slots
    is an overflow that reports how many are needed; a field along the
    track direction (no transverse momentum) scans a straight line."""
    from detray_b200 import abi, tracks
    det = oracle.build_toy()
    trk = tracks.toy_tracks(4, seed=54, pt_range=(5.0, 10.0))
    trk[:, 0] = [0.0, 0.0, 1e5, 0.0, 0.0, 0.0, 1.0, 0.1]  # far outside
    ref = oracle.helix_scan(det, B, trk, 1e-3, capacity=4)
    got = core_scan(core_host, oracle, det.desc, trk, 1e-3, capacity=4)
    assert ref["status"][0] == abi.SCAN_EMPTY
    assert np.all(ref["status"][1:] == abi.SCAN_OVERFLOW)
    assert np.all(ref["n_hits"][1:] > 4)
    assert np.array_equal(ref["status"], got["status"])
    assert np.array_equal(ref["n_hits"], got["n_hits"])
    # straight line along the field axis through the beam pipe
    line = np.array([[0.0], [0.0], [0.0], [0.0], [0.0], [0.0], [1.0], [0.5]])
    ref = oracle.helix_scan(det, B, line, 1e-3)
    got = core_scan(core_host, oracle, det.desc, line, 1e-3)
    assert_scans_match(ref, got, 1e-9)


def core_validate(core_host, scan, nav, max_records, path_tol=0.1):
    n = len(scan["status"])
    missed = np.zeros(n, dtype=np.uint32)
    extra = np.zeros(n, dtype=np.uint32)
    rc = core_host.core_host_validate(
        C.c_uint64(n), *[C.c_void_p(scan[k].ctypes.data) for k in (
            "status", "n_hits", "barcode", "path", "volume_link")],
        C.c_void_p(nav["status"].ctypes.data),
        C.c_void_p(nav["n_records"].ctypes.data),
        C.c_void_p(nav["rec_barcode"].ctypes.data),
        C.c_void_p(nav["rec_path"].ctypes.data), C.c_uint32(max_records),
        C.c_double(path_tol), C.c_void_p(missed.ctypes.data),
        C.c_void_p(extra.ctypes.data))
    assert rc == 0
    return missed, extra


@pytest.mark.parametrize("kind", ["toy", "wire_cells"])
def test_navigation_validation_host(core_host, oracle, kind):
    """The caching navigator (host build, fp64, no material so the track
    stays on its helix) reaches every surface the helix crosses and no
    other; a record taken out of the trace is reported as a hole and a
    foreign one as an extra surface."""
    from detray_b200 import abi, tracks
    from tests.test_core_host_parity import run_core
    if kind == "toy":
        det = oracle.build_toy()
        trk = tracks.toy_tracks(60, seed=55, pt_range=(1.0, 100.0))
    else:
        det = oracle.build_wire_chamber(square_cells=True)
        trk = tracks.toy_tracks(100, seed=56, pt_range=(1.0, 100.0),
                                eta_range=(-1.0, 1.0), vertex_sigma=(0, 0, 0))
    cfg = abi.make_config(max_records=128, search_window=(3, 3),
                          use_material_interactor=0,
                          estimate_scattering_noise=0, record_all_surfaces=1)
    nav = run_core(core_host, oracle, det.desc, cfg, trk, 8)
    scan = core_scan(core_host, oracle, det.desc, trk, 1e-3)
    missed, extra = core_validate(core_host, scan, nav, cfg.max_records)
    good = (missed == 0) & (extra == 0)
    assert good.mean() >= 0.95, (missed, extra)
    # plant a hole and a foreign surface in the records of a good track
    t = int(np.nonzero(good & (nav["n_records"] > 3))[0][0])
    nav2 = {k: v.copy() for k, v in nav.items()}
    sens = [k for k in range(nav["n_records"][t])
            if (int(nav["rec_barcode"][k, t]) >> 48) & 0xf == 1]
    k = sens[0]
    n_rec = nav["n_records"][t]
    for f in ("rec_barcode", "rec_path"):
        nav2[f][k:n_rec - 1, t] = nav[f][k + 1:n_rec, t]
    nav2["n_records"][t] = n_rec - 1
    m2, e2 = core_validate(core_host, scan, nav2, cfg.max_records)
    assert m2[t] == 1 and e2[t] == 0
    nav2 = {k2: v.copy() for k2, v in nav.items()}
    nav2["rec_barcode"][k, t] = nav["rec_barcode"][k, t] + (1 << 27)
    m3, e3 = core_validate(core_host, scan, nav2, cfg.max_records)
    assert m3[t] == 1 and e3[t] == 1
