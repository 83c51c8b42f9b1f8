"""GPU parity: the sm_100a propagator against the reference oracle (the
reference's own fp64 CPU propagator), through the C ABI.

Tolerances (fp32 device arithmetic against the fp64 oracle):
  surface sequences: equal for all but <= 0.1 % of the tracks (fp32 paths
      grazing a mask edge may legitimately cross a different surface);
  bound parameters at every transported surface:
      loc0/loc1  |d| <= 2e-3 + 1e-4 |x|   (mm, or rad for cylinder phi)
      phi/theta  |d| <= 2e-5 + 1e-4 |x|   (rad)
      q/p        |d| <= 1e-7 + 1e-4 |x|   (e/GeV)
      time       |d| <= 1e-6
  covariance: |dC_ij| / sqrt(C_ii C_jj) <= 1e-3.
"""
import numpy as np
import pytest

from tests.parity import compare

pytestmark = pytest.mark.gpu

TOL_ABS = {"loc0": 2e-3, "loc1": 2e-3, "phi": 2e-5, "theta": 2e-5,
           "qop": 1e-7, "time": 1e-6}
TOL_REL = 1e-4
COV_REL = 1e-3


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _run_device(torch, det, field, cfg, trk, method=0, **launch):
    from detray_b200 import propagator
    dev = torch.tensor(trk, dtype=torch.float32, device="cuda")
    lc = propagator.make_launch(method=method, **launch)
    res = propagator.propagate(cfg, det, field, dev, launch=lc)
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in res.tensors.items()}
    out["rec_barcode"] = out["rec_barcode"].view(np.uint64)
    return out


def _setup(kind):
    from detray_b200 import abi, geometry, propagator, tracks
    from detray_b200.units import T
    if kind == "telescope":
        tables = geometry.load_geometry("telescope_10x1m_300um")
        cfg = abi.make_config(max_records=16)
        trk = tracks.telescope_tracks(10000, seed=11)
    elif kind.startswith("wire"):
        tables = geometry.load_geometry(kind)
        cfg = abi.make_config(max_records=64, search_window=(3, 3),
                              estimate_scattering_noise=0)
        trk = tracks.toy_tracks(20000, seed=13, pt_range=(0.1, 100.0),
                                eta_range=(-1.0, 1.0), vertex_sigma=(0, 0, 0))
    else:
        tables = geometry.load_geometry("toy_4brl_7edc_maps" if kind == "toy_maps"
                                        else "toy_4brl_7edc")
        cfg = abi.make_config(max_records=32, search_window=(3, 3))
        trk = tracks.toy_tracks(20000, seed=12)
    det = propagator.Detector(tables)
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T))
    return det, field, cfg, trk


def _oracle_detector(oracle, kind):
    if kind == "telescope":
        return oracle.build_telescope()
    if kind.startswith("wire"):
        return oracle.build_wire_chamber(square_cells=kind.endswith("cells"))
    return oracle.build_toy(use_material_maps=kind == "toy_maps")


@pytest.mark.parametrize("kind", ["telescope", "toy", "toy_maps",
                                  "wire_chamber_10l_cells",
                                  "wire_chamber_10l_straws"])
def test_device_vs_oracle(torch_cuda, oracle, kind):
    """Both launch forms (plain; persistent, round-based, sorted) against the
    same oracle run."""
    det, field, cfg, trk = _setup(kind)
    ref_det = _oracle_detector(oracle, kind)
    ref = oracle.propagate(ref_det, field.spec, cfg, trk)
    for method, sort in ((0, 0), (1, 1)):
        got = _run_device(torch_cuda, det, field, cfg, trk, method=method,
                          sort_tracks=sort)
        summary = compare(ref, got, max_seq_mismatch_frac=1e-3,
                          tol_abs=TOL_ABS, tol_rel=TOL_REL, cov_rel=COV_REL)
        print(kind, method, summary)


@pytest.mark.parametrize("eloss_gradient", [0, 1])
def test_device_volume_material_vs_oracle(torch_cuda, oracle,
                                          eloss_gradient):
    """Telescope (config 1's 10 000 tracks) whose volume is filled with
    cesium iodide: energy loss in every RK stage, and with
    use_eloss_gradient its derivative in the transport Jacobian, on both
    launch forms against the fp64 oracle built with the same volume
    material."""
    from detray_b200 import abi, propagator, tracks
    from detray_b200.units import T
    ref_det = oracle.build_telescope(volume_material="cesium_iodide")
    det = propagator.Detector(ref_det.tables())
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T))
    cfg = abi.make_config(max_records=16, use_eloss_gradient=eloss_gradient)
    trk = tracks.telescope_tracks(10000, seed=11)
    ref = oracle.propagate(ref_det, field.spec, cfg, trk)
    for method, sort in ((0, 0), (1, 1)):
        got = _run_device(torch_cuda, det, field, cfg, trk, method=method,
                          sort_tracks=sort)
        summary = compare(ref, got, max_seq_mismatch_frac=1e-3,
                          tol_abs=TOL_ABS, tol_rel=TOL_REL, cov_rel=COV_REL)
        print("volume material", eloss_gradient, method, summary)
        # energy is lost in the volume: |q/p| at the last record above the
        # first one
        n = np.minimum(got["n_records"], cfg.max_records)
        ok = n >= 2
        cols = np.nonzero(ok)[0]
        assert np.all(np.abs(got["rec_bound"][4][n[ok] - 1, cols]) >
                      np.abs(got["rec_bound"][4][0, cols]))


def _assert_same_results(a, b, what):
    for key in ["status", "n_records", "n_steps", "n_trials",
                "n_intersections", "n_transports", "n_material",
                "path_length", "final_free"]:
        assert np.array_equal(a[key], b[key], equal_nan=a[key].dtype.kind == "f"), (what, key)
    m = int(a["n_records"].max())
    valid = np.arange(m)[:, None] < a["n_records"][None, :]
    assert np.array_equal(a["rec_barcode"][:m][valid],
                          b["rec_barcode"][:m][valid]), (what, "rec_barcode")
    for key in ["rec_bound", "rec_cov"]:
        assert np.array_equal(a[key][:, :m][:, valid],
                              b[key][:, :m][:, valid]), (what, key)
    assert np.array_equal(a["rec_path"][:m][valid], b["rec_path"][:m][valid])
    assert np.array_equal(a["rec_flags"][:m][valid], b["rec_flags"][:m][valid])


@pytest.mark.parametrize("kind", ["toy", "toy_map", "wire_chamber_10l_cells"])
def test_persistent_matches_plain(torch_cuda, kind):
    """The round-based phase kernels run the same per-track operations as
    the plain kernel, cut into segments (tests/test_rounds_host.py shows the
    two are bit-identical when compiled alike).  On the device the two are
    separate kernels, which the compiler may contract into fused
    multiply-adds differently, so they are compared with the oracle parity
    tolerances: same status and surface sequence for all but 0.1 % of the
    tracks, parameters and covariance within the fp32 tolerances - for few or
    many rounds (the rest finishing in the tail kernel), any step budget,
    yield rule and step-phase register budget."""
    if kind == "toy_map":
        from detray_b200 import abi, fields, geometry, propagator, tracks
        det = propagator.Detector(geometry.load_geometry("toy_4brl_7edc"))
        field = propagator.Field.grid(fields.solenoid_map())
        cfg = abi.make_config(max_records=32, search_window=(3, 3),
                              estimate_scattering_noise=0)
        trk = tracks.toy_tracks(20000, seed=31, pt_range=(0.1, 100.0))
    else:
        det, field, cfg, trk = _setup(kind)
    a = _run_device(torch_cuda, det, field, cfg, trk, method=0)
    for launch in [dict(sort_tracks=1),
                   dict(sort_tracks=1, ctas_per_sm=3),
                   dict(sort_tracks=0, rounds=5, steps_per_round=3,
                        yield_lanes=30, ctas_per_sm=5),
                   dict(sort_tracks=1, rounds=400, steps_per_round=64,
                        yield_lanes=1)]:
        b = _run_device(torch_cuda, det, field, cfg, trk, method=1, **launch)
        s = compare(a, b, max_seq_mismatch_frac=1e-3, tol_abs=TOL_ABS,
                    tol_rel=TOL_REL, cov_rel=COV_REL)
        print(kind, launch, s)


def test_persistent_runs_are_reproducible(torch_cuda):
    """The same launch twice: bit-identical results (the work queues are
    built in slot order, so the scheduling of the warps does not change any
    track's arithmetic)."""
    det, field, cfg, trk = _setup("toy")
    a = _run_device(torch_cuda, det, field, cfg, trk, method=1, sort_tracks=1)
    b = _run_device(torch_cuda, det, field, cfg, trk, method=1, sort_tracks=1,
                    rounds=17, steps_per_round=5)
    _assert_same_results(a, b, "reproducible")


def test_host_api_equals_device_api(torch_cuda):
    """dprop_propagate_host (host buffers, copies inside) gives the same
    records as dprop_propagate on device buffers."""
    from detray_b200 import propagator
    det, field, cfg, trk = _setup("telescope")
    a = _run_device(torch_cuda, det, field, cfg, trk)
    b = propagator.propagate_host(cfg, det, field, trk)
    assert np.array_equal(a["status"], b["status"])
    assert np.array_equal(a["n_records"], b["n_records"])
    m = int(a["n_records"].max())
    assert np.array_equal(a["rec_barcode"][:m], b["rec_barcode"][:m].view(np.uint64))
    assert np.allclose(a["rec_bound"][:, :m], b["rec_bound"][:, :m], atol=0, rtol=0)


def test_sorted_order_equals_input_order(torch_cuda):
    """Processing tracks in direction order changes only which tracks share
    a warp; with either launch form every track's result, written at its
    input position, is bit-identical to the same form in input order."""
    det, field, cfg, trk = _setup("toy")
    for method in (0, 1):
        a = _run_device(torch_cuda, det, field, cfg, trk, method=method,
                        sort_tracks=0)
        b = _run_device(torch_cuda, det, field, cfg, trk, method=method,
                        sort_tracks=1)
        _assert_same_results(a, b, ("sorted", method))


def test_empty_batch_and_invalid_arguments(torch_cuda):
    """n = 0 is a no-op; NULL detector / bad config are rejected with an
    error status, nothing is launched."""
    import ctypes as C

    from detray_b200 import abi, propagator
    det, field, cfg, trk = _setup("telescope")
    dev = torch_cuda.zeros((8, 0), dtype=torch_cuda.float32, device="cuda")
    res = propagator.alloc_device_results(0, cfg.max_records, "cuda")
    lib = propagator.load_library()
    ts = propagator.tracks_struct(torch_cuda.zeros((8, 1), device="cuda"))
    rc = lib.dprop_propagate(C.byref(cfg), None, det.handle, field.handle,
                             C.byref(ts), C.byref(res.struct), 0, None)
    assert rc == abi.DPROP_OK
    rc = lib.dprop_propagate(C.byref(cfg), None, None, field.handle,
                             C.byref(ts), C.byref(res.struct), 1, None)
    assert rc == abi.DPROP_E_INVALID
    # the energy-loss gradient without volume material: accepted (its terms
    # are identity there)
    eg = abi.make_config(max_records=16, use_eloss_gradient=1)
    one = torch_cuda.tensor(trk[:, :1], dtype=torch_cuda.float32,
                            device="cuda")
    ts1 = propagator.tracks_struct(one)
    res1 = propagator.alloc_device_results(1, eg.max_records, "cuda")
    rc = lib.dprop_propagate(C.byref(eg), None, det.handle, field.handle,
                             C.byref(ts1), C.byref(res1.struct), 1, None)
    assert rc == abi.DPROP_OK


def test_device_in_field_map_vs_oracle(torch_cuda, oracle):
    """Config-3 style: toy detector in the finite-solenoid field map,
    pT 0.1-100 GeV, direction-sorted launch."""
    from detray_b200 import abi, fields, geometry, propagator, tracks
    fmap = fields.solenoid_map()
    det = propagator.Detector(geometry.load_geometry("toy_4brl_7edc"))
    field = propagator.Field.grid(fmap)
    cfg = abi.make_config(max_records=32, search_window=(3, 3),
                          estimate_scattering_noise=0)
    trk = tracks.toy_tracks(20000, seed=31, pt_range=(0.1, 100.0))
    ref = oracle.propagate(oracle.build_toy(), fmap, cfg, trk)
    dev = torch_cuda.tensor(trk, dtype=torch_cuda.float32, device="cuda")
    res = propagator.propagate(cfg, det, field, dev,
                               launch=propagator.make_launch(sort_tracks=1))
    torch_cuda.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in res.tensors.items()}
    got["rec_barcode"] = got["rec_barcode"].view(np.uint64)
    s = compare(ref, got, max_seq_mismatch_frac=1e-3, tol_abs=TOL_ABS,
                tol_rel=TOL_REL, cov_rel=COV_REL)
    print("field map", s)


def test_device_loopers_end_cleanly(torch_cuda):
    """Low-pT loopers in the field map, with and without energy loss: every
    track ends by the path limit, by leaving, by losing its surfaces or by
    stopping (non-finite) - never by the iteration budget."""
    from detray_b200 import abi, fields, geometry, propagator, tracks
    fmap = fields.solenoid_map()
    det = propagator.Detector(geometry.load_geometry("toy_4brl_7edc"))
    field = propagator.Field.grid(fmap)
    trk = tracks.toy_tracks(4096, seed=22, pt_range=(0.02, 0.06),
                            eta_range=(-1.0, 1.0))
    dev = torch_cuda.tensor(trk, dtype=torch_cuda.float32, device="cuda")
    for material in (0, 1):
        cfg = abi.make_config(max_records=16, search_window=(3, 3),
                              estimate_scattering_noise=0,
                              use_material_interactor=material)
        res = propagator.propagate(cfg, det, field, dev,
                                   launch=propagator.make_launch(sort_tracks=1))
        torch_cuda.cuda.synchronize()
        st = res.tensors["status"].cpu().numpy()
        assert not (st == abi.TRK_MAX_ITER).any()
        assert (st == abi.TRK_PATH_LIMIT).sum() > 0
        if material:
            assert (st == abi.TRK_NONFINITE).sum() > 0


@pytest.mark.parametrize("method", [0, 1], ids=["plain", "persistent"])
def test_host_api_jagged_equals_device_api(torch_cuda, method):
    """The pipelined host path returning jagged records (several chunks on
    their own streams, the persistent method's chunks staggered) gives the
    same records as the device API with the same method."""
    from detray_b200 import abi, geometry, propagator, tracks
    from detray_b200.units import T
    det = propagator.Detector(geometry.load_geometry("toy_4brl_7edc"))
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T))
    cfg = abi.make_config(max_records=24, search_window=(3, 3))
    trk = tracks.toy_tracks(600_000, seed=41)  # 3 chunks
    a = _run_device(torch_cuda, det, field, cfg, trk, method=method,
                    sort_tracks=1)
    lc = propagator.make_launch(method=method, sort_tracks=1)
    b = propagator.propagate_host(cfg, det, field, trk, launch=lc, jagged=True)
    for key in ["status", "n_records", "n_trials", "path_length"]:
        assert np.array_equal(a[key], b[key]), key
    off = b["rec_offsets"]
    cnt = np.minimum(a["n_records"], cfg.max_records)
    assert np.array_equal(np.diff(off), cnt)
    k = np.arange(cfg.max_records)[:, None]
    valid = k < cnt[None, :]
    # slot-major (k, t) -> jagged index off[t] + k
    idx = (off[:-1][None, :] + k)[valid]
    assert np.array_equal(a["rec_barcode"][valid], b["rec_barcode"][idx].view(np.uint64))
    for i in range(6):
        assert np.array_equal(a["rec_bound"][i][valid], b["rec_bound"][i][idx])
    for i in range(21):
        assert np.array_equal(a["rec_cov"][i][valid], b["rec_cov"][i][idx])


def test_graph_replay_and_autotune(torch_cuda):
    """A propagate call captured into a CUDA graph and replayed gives the
    same results as the direct launch, plain and persistent (whose slot
    arrays and work queues the graph keeps after the sort's scratch); the
    autotuner returns one of its candidates and times all of them."""
    from detray_b200 import abi, propagator
    det, field, cfg, trk = _setup("toy")
    a = _run_device(torch_cuda, det, field, cfg, trk, method=0)
    dev = torch_cuda.tensor(trk, dtype=torch_cuda.float32, device="cuda")
    res = propagator.alloc_device_results(dev.shape[1], cfg.max_records, "cuda")
    for method, occ in ((abi.METHOD_PLAIN, 8), (abi.METHOD_PLAIN, 16),
                        (abi.METHOD_PERSISTENT, 3),
                        (abi.METHOD_PERSISTENT, 4)):
        lc = propagator.make_launch(method=method, sort_tracks=1, use_graph=1,
                                    ctas_per_sm=occ)
        for _ in range(3):  # capture, then replays
            res.tensors["status"].fill_(255)
            propagator.propagate(cfg, det, field, dev, results=res, launch=lc)
            torch_cuda.cuda.synchronize()
            b = {k: v.cpu().numpy() for k, v in res.tensors.items()}
            assert np.array_equal(a["status"], b["status"])
            assert np.array_equal(a["n_records"], b["n_records"])
            assert np.array_equal(a["path_length"], b["path_length"])
    lc, times = propagator.autotune(cfg, det, field, dev)
    assert lc.method in (abi.METHOD_PLAIN, abi.METHOD_PERSISTENT)
    if lc.method == abi.METHOD_PLAIN:
        assert lc.ctas_per_sm in (8, 12, 16)
        assert lc.block_size in (128, 256)
    else:
        assert lc.ctas_per_sm in (3, 4, 5)
        assert lc.yield_lanes in (8, 12, 16) and lc.rounds > 0
        assert lc.sort_interval in (0, 1, 2)
    chosen = ({0: "plain", 1: "persistent"}[lc.method], lc.block_size,
              lc.ctas_per_sm, lc.sort_tracks, lc.steps_per_round,
              lc.yield_lanes, lc.rounds, lc.sort_interval)
    assert chosen in propagator.AUTOTUNE_CANDIDATES
    assert len(times) == len(propagator.AUTOTUNE_CANDIDATES)
    assert all(t > 0 for t in times)
    # releasing the cached graphs and scratch: the next calls capture and
    # allocate again and give the same results
    propagator.release_cache()
    for method in (abi.METHOD_PLAIN, abi.METHOD_PERSISTENT):
        lc = propagator.make_launch(method=method, sort_tracks=1, use_graph=1)
        res.tensors["status"].fill_(255)
        propagator.propagate(cfg, det, field, dev, results=res, launch=lc)
        torch_cuda.cuda.synchronize()
        assert np.array_equal(a["status"], res.tensors["status"].cpu().numpy())
        assert np.array_equal(a["path_length"],
                              res.tensors["path_length"].cpu().numpy())
    propagator.release_cache()


@pytest.mark.parametrize("n", [1, 31, 33, 4095, 4097])
def test_persistent_small_and_ragged_batches(torch_cuda, n):
    """Batch sizes around the warp (32) and queue-tile (4096) boundaries:
    the round-based method, fp32 (graph and direct) and fp64, gives the
    plain kernel's surfaces and statuses."""
    from detray_b200 import abi, propagator
    det, field, cfg, trk = _setup("toy")
    trk = np.ascontiguousarray(trk[:, :n])
    for dtype, prec in ((torch_cuda.float32, 0), (torch_cuda.float64, 8)):
        dev = torch_cuda.tensor(trk, dtype=dtype, device="cuda")

        def run(**kw):
            res = propagator.propagate(cfg, det, field, dev,
                                       launch=propagator.make_launch(
                                           precision=prec, **kw))
            torch_cuda.cuda.synchronize()
            out = {k: v.cpu().numpy() for k, v in res.tensors.items()}
            return out

        a = run(sort_tracks=1)
        forms = [dict(method=abi.METHOD_PERSISTENT, sort_tracks=1),
                 dict(method=abi.METHOD_PERSISTENT, sort_tracks=0)]
        if prec == 0:
            forms.append(dict(method=abi.METHOD_PERSISTENT, sort_tracks=1,
                              use_graph=1))
        for kw in forms:
            b = run(**kw)
            assert np.array_equal(a["status"], b["status"]), kw
            assert np.array_equal(a["n_records"], b["n_records"]), kw
            m = int(a["n_records"].max())
            valid = np.arange(m)[:, None] < a["n_records"][None, :]
            assert np.array_equal(a["rec_barcode"][:m][valid],
                                  b["rec_barcode"][:m][valid]), kw


def test_launch_shape_does_not_change_results(torch_cuda):
    """Block size (plain) and the volume re-sort interval (persistent) only
    reorder the work: every output is bit-identical to the default launch
    of the same method, under a graph and without."""
    from detray_b200 import abi, fields, propagator
    det, _, cfg, trk = _setup("toy")
    field = propagator.Field.grid(fields.solenoid_map())
    dev = torch_cuda.tensor(trk, dtype=torch_cuda.float32, device="cuda")

    def run(**kw):
        res = propagator.propagate(cfg, det, field, dev,
                                   launch=propagator.make_launch(**kw))
        torch_cuda.cuda.synchronize()
        return {k: v.cpu().numpy() for k, v in res.tensors.items()}

    def same(a, b):
        for k in a:
            assert np.array_equal(a[k], b[k], equal_nan=True), k

    base = run(method=abi.METHOD_PLAIN, sort_tracks=1, ctas_per_sm=16)
    for blk in (32, 64, 96, 256):
        same(base, run(method=abi.METHOD_PLAIN, sort_tracks=1,
                       ctas_per_sm=16, block_size=blk))
    base = run(method=abi.METHOD_PERSISTENT, sort_tracks=1, ctas_per_sm=4)
    for si, graph in ((1, 0), (2, 1), (3, 0), (1, 1)):
        same(base, run(method=abi.METHOD_PERSISTENT, sort_tracks=1,
                       ctas_per_sm=4, sort_interval=si, use_graph=graph,
                       steps_per_round=4))
    # the tail threshold only decides in which round the last tracks run
    # to their end (1: after all rounds; n: in the first round)
    n = trk.shape[1]
    for tail in (1, n // 8, n, 10 * n):
        same(base, run(method=abi.METHOD_PERSISTENT, sort_tracks=1,
                       ctas_per_sm=4, tail_tracks=tail))
    # wire surfaces (the exact-cycle search state travels with the slots)
    det, field, cfg, trk = _setup("wire_chamber_10l_cells")
    dev = torch_cuda.tensor(trk, dtype=torch_cuda.float32, device="cuda")
    base = run(method=abi.METHOD_PERSISTENT, sort_tracks=1, ctas_per_sm=3)
    same(base, run(method=abi.METHOD_PERSISTENT, sort_tracks=1,
                   ctas_per_sm=3, sort_interval=1))
    with pytest.raises(propagator.PropagationError):
        run(method=abi.METHOD_PLAIN, block_size=48)
    with pytest.raises(propagator.PropagationError):
        run(method=abi.METHOD_PLAIN, block_size=512)
    with pytest.raises(propagator.PropagationError):
        run(method=abi.METHOD_PERSISTENT, block_size=256)


@pytest.mark.parametrize("kind", ["toy", "toy_maps", "wire_chamber_10l_cells"])
def test_fp64_device_vs_oracle(torch_cuda, oracle, kind):
    """dprop_launch.precision = 8: the propagation core in double on the
    GPU (the reference's full-fp64 build) against the fp64 oracle.  Only the
    device math library's last bits differ from the host's: same surfaces
    except <= 0.01 % of tracks, parameters to ~1e-9."""
    from detray_b200 import propagator
    det, field, cfg, trk = _setup(kind)
    ref_det = _oracle_detector(oracle, kind)
    ref = oracle.propagate(ref_det, field.spec, cfg, trk)
    dev = torch_cuda.tensor(trk, dtype=torch_cuda.float64, device="cuda")
    tight = {"loc0": 1e-6, "loc1": 1e-6, "phi": 1e-9, "theta": 1e-9,
             "qop": 1e-12, "time": 1e-9}
    # the plain kernel and the round-based phase kernels in double
    for kw in (dict(), dict(method=1), dict(method=1, ctas_per_sm=3)):
        lc = propagator.make_launch(sort_tracks=1, precision=8, **kw)
        res = propagator.propagate(cfg, det, field, dev, launch=lc)
        torch_cuda.cuda.synchronize()
        got = {k: v.cpu().numpy() for k, v in res.tensors.items()}
        got["rec_barcode"] = got["rec_barcode"].view(np.uint64)
        assert res.tensors["rec_bound"].dtype == torch_cuda.float64
        s = compare(ref, got, max_seq_mismatch_frac=1e-4, tol_abs=tight,
                    tol_rel=1e-8, cov_rel=1e-6)
        print(kind, kw, s)
    with pytest.raises(propagator.PropagationError):
        propagator.propagate(cfg, det, field, dev, launch=propagator.make_launch(
            precision=8, method=1, ctas_per_sm=4))
