"""CPU parity of the propagation core (test-only host build, tests/native)
against the reference oracle.  In double precision the core follows the
reference operation for operation: every surface sequence must match and the
recorded parameters agree to ~1e-7.  In float precision at most 0.1 % of the
tracks may cross a different surface (grazing a mask edge)."""
import ctypes as C

import numpy as np
import pytest

from tests.parity import compare

T = 0.000299792458


def run_core(core_host, oracle, det_desc, cfg, trk, precision_bytes):
    n = trk.shape[1]
    res, r = oracle.alloc_results(n, cfg.max_records)
    trk = np.ascontiguousarray(trk)
    ptrs = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    b = (C.c_double * 3)(0.0, 0.0, 2.0 * T)
    rc = core_host.core_host_propagate(precision_bytes, C.byref(det_desc), 0,
                                       b, None, None, None, None,
                                       C.byref(cfg), ptrs, C.c_uint64(n),
                                       C.byref(r))
    assert rc == 0, core_host.core_host_last_error()
    return res


TIGHT = {"loc0": 1e-7, "loc1": 1e-7, "phi": 1e-9, "theta": 1e-9,
         "qop": 1e-12, "time": 1e-12}
FP32 = {"loc0": 2e-3, "loc1": 2e-3, "phi": 2e-5, "theta": 2e-5,
        "qop": 1e-7, "time": 1e-6}


@pytest.mark.parametrize("kind,n", [("telescope", 1000), ("toy", 3000),
                                    ("toy_maps", 3000)])
def test_core_f64_matches_reference(core_host, oracle, kind, n):
    """toy_maps: the toy detector with the builder's material maps on its
    portals (a slab per bin, looked up at the bound local position)."""
    from detray_b200 import abi, tracks
    if kind == "telescope":
        det = oracle.build_telescope()
        cfg = abi.make_config(max_records=16)
        trk = tracks.telescope_tracks(n, seed=3)
    else:
        det = oracle.build_toy(use_material_maps=kind == "toy_maps")
        cfg = abi.make_config(max_records=32, search_window=(3, 3))
        trk = tracks.toy_tracks(n, seed=4)
    ref = oracle.propagate(det, {"kind": "const", "b": (0, 0, 2 * T)}, cfg, trk)
    got = run_core(core_host, oracle, det.desc, cfg, trk, 8)
    s = compare(ref, got, max_seq_mismatch_frac=0.0, tol_abs=TIGHT,
                tol_rel=1e-7, cov_rel=1e-5)
    assert s["seq_mismatch"] == 0 and s["status_mismatch"] == 0


def test_core_f32_within_tolerance(core_host, oracle):
    from detray_b200 import abi, tracks
    det = oracle.build_toy()
    cfg = abi.make_config(max_records=32, search_window=(3, 3))
    trk = tracks.toy_tracks(3000, seed=5)
    ref = oracle.propagate(det, {"kind": "const", "b": (0, 0, 2 * T)}, cfg, trk)
    got = run_core(core_host, oracle, det.desc, cfg, trk, 4)
    compare(ref, got, max_seq_mismatch_frac=1e-3, tol_abs=FP32, tol_rel=1e-4,
            cov_rel=1e-3)


def test_core_noise_estimation_and_no_material(core_host, oracle):
    """Actor-chain switches: scattering-noise tolerance on (the reference
    default) and the material interactor off."""
    from detray_b200 import abi, tracks
    det = oracle.build_toy()
    trk = tracks.toy_tracks(1000, seed=6)
    for kw in [dict(estimate_scattering_noise=1),
               dict(estimate_scattering_noise=0, use_material_interactor=0),
               dict(do_covariance_transport=0, estimate_scattering_noise=0)]:
        cfg = abi.make_config(max_records=32, search_window=(3, 3), **kw)
        ref = oracle.propagate(det, {"kind": "const", "b": (0, 0, 2 * T)},
                               cfg, trk)
        got = run_core(core_host, oracle, det.desc, cfg, trk, 8)
        tight_cov = 1e-5 if kw.get("do_covariance_transport", 1) else 1e9
        s = compare(ref, got, max_seq_mismatch_frac=0.0, tol_abs=TIGHT,
                    tol_rel=1e-7, cov_rel=tight_cov)
        assert s["seq_mismatch"] == 0, kw


WIRE = {"wire_chamber_10l_cells": True, "wire_chamber_10l_straws": False}


@pytest.mark.parametrize("name", ["toy_4brl_7edc", "toy_4brl_7edc_maps",
                                  "telescope_10x1m_300um", *WIRE])
def test_committed_geometries_match_reference_builders(oracle, name):
    """The .npz geometries the product ships are byte-identical to the
    tables the reference's own builders produce through dprop::flatten."""
    from detray_b200 import geometry
    if name.startswith("toy"):
        det = oracle.build_toy(use_material_maps=name.endswith("maps"))
    elif name.startswith("telescope"):
        det = oracle.build_telescope()
    else:
        det = oracle.build_wire_chamber(square_cells=WIRE[name])
    ref = det.tables()
    got = geometry.load_geometry(name)
    for key, _ in geometry.TABLES:
        assert ref[key].tobytes() == got[key].tobytes(), key


@pytest.mark.parametrize("square", [True, False])
def test_core_f64_matches_reference_wire_chamber(core_host, oracle, square):
    """Line surfaces (drift cells / straw tubes), material rods on the wires
    and grids with several surfaces per bin: same surfaces and parameters
    as the reference in double precision, loopers included."""
    from detray_b200 import abi, tracks
    det = oracle.build_wire_chamber(square_cells=square)
    cfg = abi.make_config(max_records=64, search_window=(3, 3),
                          estimate_scattering_noise=0)
    trk = tracks.toy_tracks(1500, seed=5, pt_range=(0.1, 100.0),
                            eta_range=(-1.0, 1.0), vertex_sigma=(0, 0, 0))
    ref = oracle.propagate(det, {"kind": "const", "b": (0, 0, 2 * T)}, cfg, trk)
    assert ref["n_records"].mean() > 8
    got = run_core(core_host, oracle, det.desc, cfg, trk, 8)
    s = compare(ref, got, max_seq_mismatch_frac=0.0, tol_abs=TIGHT,
                tol_rel=1e-7, cov_rel=1e-5)
    assert s["seq_mismatch"] == 0 and s["status_mismatch"] == 0


def test_material_map_tables_are_validated(core_host):
    """Material-map tables that point outside the slabs, at a rod, at a
    navigation grid, or carry an unknown material kind are rejected when the
    detector is read, before any track runs."""
    from detray_b200 import abi, geometry, tracks
    base = geometry.load_geometry("toy_4brl_7edc_maps")
    cfg = abi.make_config(max_records=8)
    trk = tracks.toy_tracks(4, seed=1)
    res, r = _alloc(4, cfg.max_records)
    mapped = np.nonzero(base["surfaces"]["material_kind"] == 1)[0]
    first_map = int(base["surfaces"]["material"][mapped[0]])
    first_bin = int(base["grids"]["bin_offset"][first_map])
    nav_grid = int(np.nonzero(base["grids"]["kind"] == abi.GRID_CYLINDER)[0][0])

    def run(tables):
        desc = geometry.Descriptor(tables)
        ptrs = (C.c_void_p * 8)(*[np.ascontiguousarray(trk[i]).ctypes.data
                                  for i in range(8)])
        b = (C.c_double * 3)(0.0, 0.0, 2.0 * T)
        return core_host.core_host_propagate(8, C.byref(desc.desc), 0, b, None,
                                             None, None, None, C.byref(cfg),
                                             ptrs, C.c_uint64(4), C.byref(r))

    assert run(base) == 0
    bad = []
    t = {k: v.copy() for k, v in base.items()}
    t["grid_bins"][first_bin] = len(t["slabs"])
    bad.append(t)
    t = {k: v.copy() for k, v in base.items()}
    t["slabs"]["kind"][t["grid_bins"][first_bin]] = abi.MATERIAL_ROD
    bad.append(t)
    t = {k: v.copy() for k, v in base.items()}
    t["surfaces"]["material"][mapped[0]] = nav_grid
    bad.append(t)
    t = {k: v.copy() for k, v in base.items()}
    t["surfaces"]["material_kind"][mapped[0]] = 2
    bad.append(t)
    t = {k: v.copy() for k, v in base.items()}
    t["grids"]["kind"][first_map] = 6
    bad.append(t)
    for i, tables in enumerate(bad):
        assert run(tables) != 0, i
        assert core_host.core_host_last_error(), i


def _alloc(n, max_records):
    from oracle import ref_oracle
    return ref_oracle.alloc_results(n, max_records)


@pytest.mark.parametrize("material", ["cesium_iodide", "iron", "silicon"])
@pytest.mark.parametrize("eloss_gradient", [0, 1])
def test_core_f64_volume_material(core_host, oracle, material,
                                  eloss_gradient):
    """A telescope whose volume is filled with a homogeneous material
    (tel_det_config::volume_material): the stepper loses energy along every
    step (d(q/p)/ds per RK stage from the Bethe-Bloch stopping power) and,
    with use_eloss_gradient, carries d(q/p)/d(q/p0) into the transport
    Jacobian (rk_stepper.hpp:146-231, 760-800).  fp64 host core against the
    fp64 oracle: same surfaces, parameters to ~1e-7, with and without the
    mean-loss stage update."""
    from detray_b200 import abi, tracks
    det = oracle.build_telescope(volume_material=material)
    assert det.desc.volumes[0].material != abi.DPROP_INVALID_INDEX
    trk = tracks.telescope_tracks(1000, seed=7)
    for mean_loss in (1, 0):
        cfg = abi.make_config(max_records=16, use_mean_loss=mean_loss,
                              use_eloss_gradient=eloss_gradient)
        ref = oracle.propagate(det, {"kind": "const", "b": (0, 0, 2 * T)},
                               cfg, trk)
        got = run_core(core_host, oracle, det.desc, cfg, trk, 8)
        s = compare(ref, got, max_seq_mismatch_frac=0.0, tol_abs=TIGHT,
                    tol_rel=1e-7, cov_rel=1e-5)
        assert s["seq_mismatch"] == 0 and s["status_mismatch"] == 0
        # the volume material takes energy: |q/p| grows along the track
        n = np.minimum(got["n_records"], cfg.max_records)
        ok = n >= 2
        last = got["rec_bound"][4][n[ok] - 1, np.nonzero(ok)[0]]
        first = got["rec_bound"][4][0, ok]
        assert np.all(np.abs(last) > np.abs(first))
