"""The allocation-free entry point dprop_propagate_noalloc.

Callers such as event-processing frameworks that own all device memory
through their own pool, or latency-bound trigger loops that may not call
cudaMalloc/cudaFree (which can synchronise the whole device), cannot let the
library allocate.  dprop_propagate_noalloc serves them: the direction-sorted
propagation with its sort scratch in a fixed array inside the library.

These tests call it through the C ABI and check, on two calls in a row with
different tracks, that it returns exactly what the allocating entry point
dprop_propagate returns for the same tracks (both run the same per-track
code, so the tolerance is zero), that it allocates no device memory, that
a batch of exactly its capacity fits, and that batches above its fixed
capacity are rejected with a clear error.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from detray_b200 import abi, geometry, propagator
    from detray_b200.units import T
    lib = propagator.load_library()
    lib.dprop_propagate_noalloc.argtypes = [
        C.POINTER(abi.Config), C.c_void_p, C.c_void_p, C.POINTER(abi.Tracks),
        C.POINTER(abi.Results), C.c_uint64, C.c_void_p]
    det = propagator.Detector(geometry.load_geometry("toy_4brl_7edc"))
    field = propagator.Field.constant((0.0, 0.0, 2.0 * T))
    cfg = abi.make_config(max_records=32, search_window=(3, 3))
    return torch, lib, det, field, cfg


def _host(res):
    return {k: v.cpu().numpy() for k, v in res.tensors.items()}


def _noalloc(torch, lib, det, field, cfg, trk_dev):
    from detray_b200 import propagator
    n = trk_dev.shape[1]
    res = propagator.alloc_device_results(n, cfg.max_records, "cuda")
    ts = propagator.tracks_struct(trk_dev)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    rc = lib.dprop_propagate_noalloc(C.byref(cfg), det.handle, field.handle,
                                     C.byref(ts), C.byref(res.struct), n,
                                     C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert rc == 0, lib.dprop_last_error().decode()
    return res, free_before - free_after


def test_noalloc_matches_allocating_entry_point(setup):
    torch, lib, det, field, cfg = setup
    from detray_b200 import propagator, tracks
    grown = []
    for call, seed in enumerate((101, 202)):
        trk = torch.tensor(tracks.toy_tracks(60_000, seed=seed),
                           dtype=torch.float32, device="cuda")
        ref = _host(propagator.propagate(
            cfg, det, field, trk,
            launch=propagator.make_launch(sort_tracks=1)))
        res, grew = _noalloc(torch, lib, det, field, cfg, trk)
        got = _host(res)
        grown.append(grew)
        for key in ["status", "n_records", "n_steps", "n_trials",
                    "path_length", "final_free", "n_intersections"]:
            assert np.array_equal(ref[key], got[key]), (call, key)
        m = int(ref["n_records"].max())
        valid = np.arange(m)[:, None] < np.minimum(ref["n_records"], 32)[None, :]
        assert np.array_equal(ref["rec_barcode"][:m][valid],
                              got["rec_barcode"][:m][valid]), call
        for key in ["rec_bound", "rec_cov"]:
            a = ref[key][:, :m][:, valid]
            b = got[key][:, :m][:, valid]
            assert np.allclose(a, b, rtol=0.0, atol=0.0), (call, key)
    # the second call runs on warm code: it must not take device memory
    assert grown[1] == 0, f"device memory shrank by {grown[1]} bytes"


def test_noalloc_takes_its_full_capacity(setup):
    """A batch of exactly DPROP_NOALLOC_MAX_TRACKS tracks fits the fixed
    scratch (sort keys, indices and the radix sort's temporary storage) and
    gives the allocating entry point's results."""
    torch, lib, det, field, cfg = setup
    from detray_b200 import propagator, tracks
    n = 262_144
    trk = torch.tensor(tracks.toy_tracks(n, seed=303), dtype=torch.float32,
                       device="cuda")
    ref = _host(propagator.propagate(
        cfg, det, field, trk, launch=propagator.make_launch(sort_tracks=1)))
    res, _ = _noalloc(torch, lib, det, field, cfg, trk)
    got = _host(res)
    for key in ["status", "n_records", "n_steps", "path_length",
                "final_free"]:
        assert np.array_equal(ref[key], got[key]), key


def test_noalloc_rejects_batches_above_capacity(setup):
    torch, lib, det, field, cfg = setup
    from detray_b200 import abi, propagator
    n = 262_144 + 1
    trk = torch.zeros((8, 1), dtype=torch.float32, device="cuda")
    res = propagator.alloc_device_results(1, cfg.max_records, "cuda")
    ts = propagator.tracks_struct(trk)
    rc = lib.dprop_propagate_noalloc(C.byref(cfg), det.handle, field.handle,
                                     C.byref(ts), C.byref(res.struct), n, None)
    assert rc == abi.DPROP_E_INVALID
    assert "262144" in lib.dprop_last_error().decode()
