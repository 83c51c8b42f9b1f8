"""The r-phi-z field map: the device lookup (host build of the core) against
the oracle's field class, the map against the analytic finite solenoid, and
the propagation through the map against the reference oracle (CPU)."""
import ctypes as C

import numpy as np
import pytest

from tests.parity import compare


@pytest.fixture(scope="module")
def solenoid():
    from detray_b200 import fields
    return fields.solenoid_map()


def _core_field(core_host, fmap, pts, precision):
    core_host.core_host_field_eval.argtypes = [
        C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
        C.POINTER(C.c_uint32), C.POINTER(C.c_float), C.POINTER(C.c_double),
        C.c_uint64, C.POINTER(C.c_double)]
    vals = np.ascontiguousarray(fmap["values"], dtype=np.float32)
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    out = np.zeros_like(pts)
    core_host.core_host_field_eval(
        precision, (C.c_double * 3)(*fmap["lo"]), (C.c_double * 3)(*fmap["hi"]),
        (C.c_uint32 * 3)(*fmap["n"]), vals.ctypes.data_as(C.POINTER(C.c_float)),
        pts.ctypes.data_as(C.POINTER(C.c_double)), pts.shape[0],
        out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def _random_points(n, seed, r_max=1600.0, z_max=3700.0):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.0, r_max, n)
    phi = rng.uniform(-np.pi, np.pi, n)
    z = rng.uniform(-z_max, z_max, n)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def test_device_lookup_matches_oracle_field(core_host, oracle, solenoid):
    pts = _random_points(20000, 1)  # includes points outside the map (clamped)
    ref = oracle.field_eval(solenoid, pts)
    got64 = _core_field(core_host, solenoid, pts, 8)
    got32 = _core_field(core_host, solenoid, pts, 4)
    scale = np.abs(ref).max()
    assert np.abs(got64 - ref).max() <= 1e-12 * scale
    # fp32 cell coordinates of points up to 3.7 m: ~1e-5 of a 20 mm cell
    assert np.abs(got32 - ref).max() <= 1e-5 * scale


def test_map_reproduces_analytic_solenoid(solenoid):
    """Between nodes, trilinear interpolation of the 20 mm map stays within
    1e-3 relative of the analytic field in the tracker volume."""
    from detray_b200 import fields
    rng = np.random.default_rng(2)
    r = rng.uniform(0.0, 600.0, 2000)
    z = rng.uniform(-2000.0, 2000.0, 2000)
    br, bz = fields.solenoid_field(r, z)
    v = solenoid["values"][:, 0, :, :].astype(np.float64)
    # bilinear (r, z) interpolation, one phi node
    fr = r / 20.0
    fz = (z + 3500.0) / 20.0
    i0 = np.floor(fr).astype(int)
    j0 = np.floor(fz).astype(int)
    ur, uz = fr - i0, fz - j0
    def interp(c):
        return ((1 - ur) * (1 - uz) * v[j0, i0, c] + ur * (1 - uz) * v[j0, i0 + 1, c]
                + (1 - ur) * uz * v[j0 + 1, i0, c] + ur * uz * v[j0 + 1, i0 + 1, c])
    b0 = np.abs(bz).max()
    assert np.abs(interp(2) - bz).max() <= 1e-3 * b0
    assert np.abs(interp(0) - br).max() <= 1e-3 * b0


def test_propagation_in_field_map_matches_reference(core_host, oracle, solenoid):
    """Config-3 style tracks (pT 0.1-100 GeV, loopers included) through the
    toy detector in the solenoid map: core (double) vs reference oracle."""
    from detray_b200 import abi, tracks
    det = oracle.build_toy()
    cfg = abi.make_config(max_records=64, search_window=(3, 3),
                          estimate_scattering_noise=0)
    trk = tracks.toy_tracks(1500, seed=21, pt_range=(0.1, 100.0))
    ref = oracle.propagate(det, solenoid, cfg, trk)
    n = trk.shape[1]
    res, r = oracle.alloc_results(n, cfg.max_records)
    vals = np.ascontiguousarray(solenoid["values"], dtype=np.float32)
    ptrs = (C.c_void_p * 8)(*[np.ascontiguousarray(trk[i]).ctypes.data
                              for i in range(8)])
    keep = [np.ascontiguousarray(trk[i]) for i in range(8)]
    ptrs = (C.c_void_p * 8)(*[k.ctypes.data for k in keep])
    rc = core_host.core_host_propagate(
        8, C.byref(det.desc), 1, (C.c_double * 3)(0, 0, 0),
        (C.c_double * 3)(*solenoid["lo"]), (C.c_double * 3)(*solenoid["hi"]),
        (C.c_uint32 * 3)(*solenoid["n"]),
        vals.ctypes.data_as(C.POINTER(C.c_float)), C.byref(cfg), ptrs,
        C.c_uint64(n), C.byref(r))
    assert rc == 0
    tight = {"loc0": 1e-6, "loc1": 1e-6, "phi": 1e-8, "theta": 1e-8,
             "qop": 1e-11, "time": 1e-12}
    s = compare(ref, res, max_seq_mismatch_frac=0.0, tol_abs=tight,
                tol_rel=1e-6, cov_rel=1e-4)
    assert s["seq_mismatch"] == 0
    assert np.array_equal(ref["status"], res["status"])


def _core_in_map(core_host, oracle, det, solenoid, cfg, trk):
    n = trk.shape[1]
    res, r = oracle.alloc_results(n, cfg.max_records)
    vals = np.ascontiguousarray(solenoid["values"], dtype=np.float32)
    keep = [np.ascontiguousarray(trk[i]) for i in range(8)]
    ptrs = (C.c_void_p * 8)(*[k.ctypes.data for k in keep])
    rc = core_host.core_host_propagate(
        8, C.byref(det.desc), 1, (C.c_double * 3)(0, 0, 0),
        (C.c_double * 3)(*solenoid["lo"]), (C.c_double * 3)(*solenoid["hi"]),
        (C.c_uint32 * 3)(*solenoid["n"]),
        vals.ctypes.data_as(C.POINTER(C.c_float)), C.byref(cfg), ptrs,
        C.c_uint64(n), C.byref(r))
    assert rc == 0
    return res


def test_stopping_muons_end_as_nonfinite(core_host, oracle, solenoid):
    """Slow muons (20-60 MeV) lose all their momentum in the silicon: the
    interactor sets q/p to the invalid maximum.  The reference then keeps
    computing with inf/NaN (undefined behaviour, it can crash), so it cannot
    serve as the oracle here; the device core must end such tracks with
    DPROP_TRK_NONFINITE and never run into its iteration budget."""
    from detray_b200 import abi, tracks
    det = oracle.build_toy()
    cfg = abi.make_config(max_records=48, search_window=(3, 3),
                          estimate_scattering_noise=0)
    trk = tracks.toy_tracks(200, seed=22, pt_range=(0.02, 0.06),
                            eta_range=(-1.0, 1.0))
    got = _core_in_map(core_host, oracle, det, solenoid, cfg, trk)
    st = got["status"]
    assert (st == abi.TRK_NONFINITE).sum() > 0
    # every track ends for a physical or navigational reason, none by
    # running into the iteration budget
    assert not (st == abi.TRK_MAX_ITER).any()
    assert not (st == abi.TRK_NOT_RUN).any()
    assert np.isfinite(got["rec_bound"][4][got["rec_flags"] & 1 > 0]).all()


def test_loopers_reach_path_limit(core_host, oracle, solenoid):
    """Low-pT loopers without energy loss curl inside the barrel until the
    5 m path limit: long tracks with more records than the capacity.  (The
    reference mis-handles the grid lookup when the tangent ray misses a
    layer's reference cylinder - undefined behaviour on curling tracks - so
    this is a robustness check of the core, in double and float.)"""
    from detray_b200 import abi, tracks
    det = oracle.build_toy()
    cfg = abi.make_config(max_records=8, search_window=(3, 3),
                          estimate_scattering_noise=0,
                          use_material_interactor=0)
    trk = tracks.toy_tracks(200, seed=22, pt_range=(0.02, 0.06),
                            eta_range=(-1.0, 1.0))
    got = _core_in_map(core_host, oracle, det, solenoid, cfg, trk)
    st = got["status"]
    assert (st == abi.TRK_PATH_LIMIT).sum() > trk.shape[1] // 5
    assert not (st == abi.TRK_MAX_ITER).any()
    assert (got["n_records"] > cfg.max_records).any()
    # the signed path length never exceeds the limit on the absolute path
    # (curling tracks also step backwards onto surfaces they overstepped)
    assert np.all(np.abs(got["path_length"]) <= 5000.0 + 1.0)


def test_field_gradient_transport_matches_reference(core_host, oracle,
                                                    solenoid):
    """use_field_gradient in the solenoid map: the transport Jacobian with
    the field's gradient (position columns from central differences of the
    field at the three RKN points) gives the reference's covariances (the
    oracle runs the reference's with-gradient rk_stepper); without it the
    covariances differ where the map varies."""
    from detray_b200 import abi, tracks
    det = oracle.build_toy()
    trk = tracks.toy_tracks(800, seed=23, pt_range=(0.5, 10.0),
                            eta_range=(-3.0, 3.0))
    tight = {"loc0": 1e-6, "loc1": 1e-6, "phi": 1e-8, "theta": 1e-8,
             "qop": 1e-11, "time": 1e-12}
    cfg = abi.make_config(max_records=32, search_window=(3, 3),
                          estimate_scattering_noise=0, use_field_gradient=1)
    ref = oracle.propagate(det, solenoid, cfg, trk)
    got = _core_in_map(core_host, oracle, det, solenoid, cfg, trk)
    s = compare(ref, got, max_seq_mismatch_frac=0.0, tol_abs=tight,
                tol_rel=1e-6, cov_rel=1e-5)
    assert s["seq_mismatch"] == 0
    cfg0 = abi.make_config(max_records=32, search_window=(3, 3),
                           estimate_scattering_noise=0)
    plain = _core_in_map(core_host, oracle, det, solenoid, cfg0, trk)
    m = (np.arange(32)[:, None] < got["n_records"][None, :]) & \
        ((got["rec_flags"] & 1) > 0)
    dcov = np.abs(plain["rec_cov"][0][m] - got["rec_cov"][0][m]) / \
        np.abs(got["rec_cov"][0][m])
    assert dcov.max() > 1e-4  # the gradient changes the transported errors
