"""Python binding of the B200 propagator over its C ABI.

Mirrors the reference's device propagation call shape
(tests/benchmarks/include/detray/benchmarks/device/cuda/
propagation_benchmark.hpp:83-93):

    det   = Detector(tables)                       # detray::get_buffer/get_data
    field = Field.constant((0, 0, 2 * unit.T))     # covfie constant field view
    res   = propagate(cfg, det, field, tracks)     # run_propagation_kernel

Device memory and streams come from PyTorch; the propagation itself is the
sm_100a library ``detray_b200/_lib/libdetray_b200.so``.  There is no CPU
fallback: if the library or a CUDA device is missing, the calls raise.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import abi
from .geometry import Descriptor

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libdetray_b200.so"

_lib = None

#: exported symbols of the C ABI (include/detray_b200/dprop.h)
ABI_SYMBOLS = [
    "dprop_abi_version", "dprop_last_error", "dprop_config_default",
    "dprop_detector_create", "dprop_detector_destroy", "dprop_detector_info",
    "dprop_field_create_const", "dprop_field_create_grid",
    "dprop_field_destroy", "dprop_propagate", "dprop_propagate_host",
    "dprop_propagate_noalloc", "dprop_autotune", "dprop_propagate_adjoint",
    "dprop_backward", "dprop_propagate_direct", "dprop_helix_scan",
    "dprop_validate_navigation", "dprop_release_cache",
]


class PropagationError(RuntimeError):
    pass


def load_library() -> C.CDLL:
    """Load the device library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise PropagationError(
            f"{LIB_PATH} not found: the CUDA library is not built "
            "(run __graft_entry__.build() or detray_b200/build.py)")
    lib = C.CDLL(str(LIB_PATH))
    lib.dprop_abi_version.restype = C.c_uint32
    lib.dprop_last_error.restype = C.c_char_p
    lib.dprop_config_default.argtypes = [C.POINTER(abi.Config)]
    lib.dprop_detector_create.argtypes = [C.POINTER(abi.DetectorDesc), C.c_int,
                                          C.POINTER(C.c_void_p)]
    lib.dprop_detector_destroy.argtypes = [C.c_void_p]
    lib.dprop_detector_info.argtypes = [C.c_void_p, C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_uint32)]
    lib.dprop_field_create_const.argtypes = [C.c_double, C.c_double,
                                             C.c_double, C.c_int,
                                             C.POINTER(C.c_void_p)]
    lib.dprop_field_create_grid.argtypes = [
        C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_uint32),
        C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_void_p)]
    lib.dprop_field_destroy.argtypes = [C.c_void_p]
    lib.dprop_propagate.argtypes = [
        C.POINTER(abi.Config), C.POINTER(abi.Launch), C.c_void_p, C.c_void_p,
        C.POINTER(abi.Tracks), C.POINTER(abi.Results), C.c_uint64, C.c_void_p]
    lib.dprop_propagate_host.argtypes = [
        C.POINTER(abi.Config), C.POINTER(abi.Launch), C.c_void_p, C.c_void_p,
        C.POINTER(abi.Tracks), C.POINTER(abi.Results), C.c_uint64]
    lib.dprop_autotune.argtypes = [
        C.POINTER(abi.Config), C.c_void_p, C.c_void_p, C.POINTER(abi.Tracks),
        C.c_uint64, C.POINTER(abi.Launch), C.POINTER(C.c_float), C.c_void_p]
    lib.dprop_propagate_adjoint.argtypes = [
        C.POINTER(abi.Config), C.POINTER(abi.Launch), C.c_void_p, C.c_void_p,
        C.POINTER(abi.Tracks), C.POINTER(abi.Results), C.POINTER(abi.Tape),
        C.c_uint64, C.c_void_p]
    lib.dprop_backward.argtypes = [
        C.POINTER(abi.Config), C.c_void_p, C.POINTER(abi.Tracks),
        C.POINTER(abi.Results), C.POINTER(abi.Tape),
        C.POINTER(abi.Gradients), C.c_uint64, C.c_void_p]
    lib.dprop_propagate_direct.argtypes = [
        C.POINTER(abi.Config), C.c_void_p, C.c_void_p, C.POINTER(abi.Tracks),
        C.POINTER(abi.Sequence), C.POINTER(abi.Results), C.c_uint64,
        C.c_void_p]
    lib.dprop_helix_scan.argtypes = [
        C.c_void_p, C.POINTER(C.c_double), C.POINTER(abi.Tracks), C.c_uint64,
        C.c_double, C.POINTER(abi.ScanResults), C.c_void_p]
    lib.dprop_validate_navigation.argtypes = [
        C.POINTER(abi.ScanResults), C.POINTER(abi.Results), C.c_uint32,
        C.c_uint32, C.c_uint64, C.c_double, C.POINTER(abi.Validation),
        C.c_void_p]
    if lib.dprop_abi_version() != abi.DPROP_ABI_VERSION:
        raise PropagationError("detray-b200 library ABI version mismatch")
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != abi.DPROP_OK:
        msg = load_library().dprop_last_error().decode()
        raise PropagationError(f"dprop status {rc}: {msg}")


def default_config(**overrides) -> abi.Config:
    """propagation::config defaults plus the actor-chain switches."""
    return abi.make_config(**overrides)


class Detector:
    """Device copy of a detector's flat tables (immutable once created)."""

    def __init__(self, tables: dict, device: int = 0):
        lib = load_library()
        self._desc = Descriptor(tables)
        self.handle = C.c_void_p()
        _check(lib.dprop_detector_create(C.byref(self._desc.desc), device,
                                         C.byref(self.handle)))
        self.device = device
        self.n_surfaces = len(self._desc.tables["surfaces"])
        self.n_volumes = len(self._desc.tables["volumes"])

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            load_library().dprop_detector_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Field:
    """Magnetic field view on the device."""

    def __init__(self, handle: C.c_void_p, spec: dict):
        self.handle = handle
        self.spec = spec

    @classmethod
    def constant(cls, b, device: int = 0) -> "Field":
        lib = load_library()
        h = C.c_void_p()
        _check(lib.dprop_field_create_const(float(b[0]), float(b[1]),
                                            float(b[2]), device, C.byref(h)))
        return cls(h, {"kind": "const", "b": tuple(float(x) for x in b)})

    @classmethod
    def grid(cls, spec: dict, device: int = 0) -> "Field":
        """spec: {"lo": (r, phi, z), "hi": ..., "n": (nr, nphi, nz),
        "values": float32 array (nz, nphi, nr, 3)}"""
        lib = load_library()
        lo = (C.c_double * 3)(*spec["lo"])
        hi = (C.c_double * 3)(*spec["hi"])
        n = (C.c_uint32 * 3)(*spec["n"])
        vals = np.ascontiguousarray(spec["values"], dtype=np.float32)
        h = C.c_void_p()
        _check(lib.dprop_field_create_grid(
            lo, hi, n, vals.ctypes.data_as(C.POINTER(C.c_float)), device,
            C.byref(h)))
        return cls(h, dict(spec, kind="grid"))

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            load_library().dprop_field_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def release_cache() -> None:
    """Free the device memory the library keeps between calls (cached CUDA
    graphs and grow-only scratch; dprop_release_cache)."""
    _check(load_library().dprop_release_cache())


def make_launch(method: int = abi.METHOD_PLAIN, block_size: int = 0,
                ctas_per_sm: int = 0, sort_tracks: int = 0,
                use_graph: int = 0, precision: int = 0,
                steps_per_round: int = 0, rounds: int = 0,
                yield_lanes: int = 0, sort_interval: int = 0,
                tail_tracks: int = 0) -> abi.Launch:
    """Launch shape; ``precision`` 8 runs the propagation in fp64 end to end
    (double track tensors and results).  steps_per_round, rounds,
    yield_lanes, sort_interval and tail_tracks shape the persistent
    (round-based) method; 0 picks the library default (sort_interval 0: no
    re-sort by volume; tail_tracks 0: n / 64)."""
    lc = abi.Launch()
    lc.method = method
    lc.block_size = block_size
    lc.ctas_per_sm = ctas_per_sm
    lc.sort_tracks = sort_tracks
    lc.use_graph = use_graph
    lc.precision = precision
    lc.steps_per_round = steps_per_round
    lc.rounds = rounds
    lc.yield_lanes = yield_lanes
    lc.sort_interval = sort_interval
    lc.tail_tracks = tail_tracks
    return lc


@dataclass
class DeviceResults:
    """Device result buffers (torch tensors) + the ABI struct pointing at
    them."""
    tensors: dict
    struct: abi.Results
    inputs: list | None = None  # input tensors a call must keep alive


def alloc_device_results(n: int, max_records: int, device="cuda",
                         with_records=True, with_cov=True,
                         dtype=None) -> DeviceResults:
    """Result buffers; floating-point fields in ``dtype`` (float32 default,
    float64 for fp64 launches)."""
    import torch
    f32 = dict(dtype=dtype or torch.float32, device=device)
    t = {
        "status": torch.empty(n, dtype=torch.uint8, device=device),
        "n_records": torch.empty(n, dtype=torch.int32, device=device),
        "n_steps": torch.empty(n, dtype=torch.int32, device=device),
        "n_trials": torch.empty(n, dtype=torch.int32, device=device),
        "path_length": torch.empty(n, **f32),
        "final_free": torch.empty((8, n), **f32),
        "n_intersections": torch.empty(n, dtype=torch.int32, device=device),
        "n_transports": torch.empty(n, dtype=torch.int32, device=device),
        "n_material": torch.empty(n, dtype=torch.int32, device=device),
    }
    r = abi.Results()
    r.n_intersections = t["n_intersections"].data_ptr()
    r.n_transports = t["n_transports"].data_ptr()
    r.n_material = t["n_material"].data_ptr()
    r.status = t["status"].data_ptr()
    r.n_records = t["n_records"].data_ptr()
    r.n_steps = t["n_steps"].data_ptr()
    r.n_trials = t["n_trials"].data_ptr()
    r.path_length = t["path_length"].data_ptr()
    for i in range(8):
        r.final_free[i] = t["final_free"][i].data_ptr()
    if with_records and max_records > 0:
        t["rec_barcode"] = torch.empty((max_records, n), dtype=torch.int64,
                                       device=device)
        t["rec_bound"] = torch.empty((6, max_records, n), **f32)
        t["rec_path"] = torch.empty((max_records, n), **f32)
        t["rec_flags"] = torch.empty((max_records, n), dtype=torch.uint8,
                                     device=device)
        r.rec_barcode = t["rec_barcode"].data_ptr()
        for i in range(6):
            r.rec_bound[i] = t["rec_bound"][i].data_ptr()
        r.rec_path = t["rec_path"].data_ptr()
        r.rec_flags = t["rec_flags"].data_ptr()
        if with_cov:
            t["rec_cov"] = torch.empty((21, max_records, n), **f32)
            for i in range(21):
                r.rec_cov[i] = t["rec_cov"][i].data_ptr()
    return DeviceResults(t, r)


def tracks_struct(trk) -> abi.Tracks:
    """ABI track pointers for a (8, n) contiguous float32 CUDA tensor or a
    (8, n) float64 host numpy array."""
    ts = abi.Tracks()
    if hasattr(trk, "data_ptr"):
        rows = [trk[i].data_ptr() for i in range(8)]
    else:
        rows = [trk[i].ctypes.data for i in range(8)]
    for i in range(3):
        ts.pos[i] = rows[i]
        ts.dir[i] = rows[4 + i]
    ts.time = rows[3]
    ts.qop = rows[7]
    return ts


def propagate(cfg: abi.Config, det: Detector, field: Field, tracks,
              results: DeviceResults | None = None, launch: abi.Launch | None = None,
              stream=None) -> DeviceResults:
    """Propagate the tracks of a (8, n) float32 CUDA tensor; stream ordered
    on ``stream`` (default: torch's current stream)."""
    import torch
    if not (hasattr(tracks, "is_cuda") and tracks.is_cuda):
        raise PropagationError("propagate() needs a CUDA tensor of tracks")
    fp64 = launch is not None and launch.precision == 8
    want = torch.float64 if fp64 else torch.float32
    if tracks.dtype != want or tracks.dim() != 2 or tracks.shape[0] != 8:
        raise PropagationError(f"tracks must be a (8, n) {want} tensor")
    tracks = tracks.contiguous()
    n = tracks.shape[1]
    if results is None:
        results = alloc_device_results(n, cfg.max_records, tracks.device,
                                       dtype=want)
    if stream is None:
        stream = torch.cuda.current_stream(tracks.device)
    ts = tracks_struct(tracks)
    lc = launch if launch is not None else make_launch()
    _check(load_library().dprop_propagate(
        C.byref(cfg), C.byref(lc), det.handle, field.handle, C.byref(ts),
        C.byref(results.struct), n, C.c_void_p(stream.cuda_stream)))
    return results


def propagate_direct(cfg: abi.Config, det: Detector, field: Field,
                     sequence, lengths, direction: int = 1, tracks=None,
                     start_barcode=None, start_bound=None,
                     results: DeviceResults | None = None,
                     stream=None) -> DeviceResults:
    """Propagate along given surface sequences with the direct navigator
    (dprop_propagate_direct).  ``sequence``: (max_length, n) int64 CUDA
    tensor of surface barcodes, e.g. ``rec_barcode`` of a propagate() run;
    ``lengths``: (n,) int32 CUDA tensor (``n_records``).  Start from the
    (8, n) float32 ``tracks`` or from bound parameters ``start_bound``
    ((6, n) float32) on the surfaces ``start_barcode`` ((n,) int64)."""
    import torch
    n = lengths.shape[0]
    dev = lengths.device
    for name, t in (("sequence", sequence), ("lengths", lengths)):
        if not (hasattr(t, "is_cuda") and t.is_cuda):
            raise PropagationError(f"{name} must be a CUDA tensor")
    if sequence.dtype != torch.int64 or sequence.dim() != 2 or \
            sequence.shape[1] != n:
        raise PropagationError("sequence must be a (max_length, n) int64 "
                               "tensor")
    if lengths.dtype != torch.int32:
        raise PropagationError("lengths must be an int32 tensor")
    sequence = sequence.contiguous()
    lengths = lengths.contiguous()
    sq = abi.Sequence()
    sq.barcodes = sequence.data_ptr() if sequence.numel() else None
    sq.length = lengths.data_ptr()
    sq.max_length = sequence.shape[0]
    sq.direction = int(direction)
    ts = None
    keep = [sequence, lengths]
    if start_barcode is not None:
        if start_bound is None or start_bound.dtype != torch.float32 or \
                tuple(start_bound.shape) != (6, n):
            raise PropagationError("start_bound must be a (6, n) float32 "
                                   "tensor")
        start_barcode = start_barcode.contiguous()
        start_bound = start_bound.contiguous()
        keep += [start_barcode, start_bound]
        sq.start_barcode = start_barcode.data_ptr()
        for i in range(6):
            sq.start_bound[i] = start_bound[i].data_ptr()
    else:
        if tracks is None or tracks.dtype != torch.float32 or \
                tuple(tracks.shape) != (8, n):
            raise PropagationError("tracks must be a (8, n) float32 tensor")
        tracks = tracks.contiguous()
        keep.append(tracks)
        ts = tracks_struct(tracks)
    if results is None:
        results = alloc_device_results(n, cfg.max_records, dev)
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    _check(load_library().dprop_propagate_direct(
        C.byref(cfg), det.handle, field.handle,
        C.byref(ts) if ts is not None else None, C.byref(sq),
        C.byref(results.struct), n, C.c_void_p(stream.cuda_stream)))
    results.inputs = keep  # alive until the caller drops the results
    return results


def helix_scan(det: Detector, b, tracks, mask_tolerance: float = 0.0,
               capacity: int = 256, stream=None) -> dict:
    """Truth intersections of every track's helix in the constant field
    ``b`` (3 components, detray units) with all surfaces of ``det``
    (dprop_helix_scan): per track the hits inside a mask and along the
    track, sorted by path and cut after the first world exit.  ``tracks``:
    (8, n) float32 or float64 CUDA tensor; the results have its precision.
    Returns CUDA tensors: status, n_hits, barcode/path/loc0/loc1/volume_link
    of shape (capacity, n)."""
    import torch
    if not (hasattr(tracks, "is_cuda") and tracks.is_cuda) or \
            tracks.dim() != 2 or tracks.shape[0] != 8 or \
            tracks.dtype not in (torch.float32, torch.float64):
        raise PropagationError("tracks must be a (8, n) float32/float64 "
                               "CUDA tensor")
    tracks = tracks.contiguous()
    n = tracks.shape[1]
    dev = tracks.device
    ft = dict(dtype=tracks.dtype, device=dev)
    out = {
        "status": torch.empty(n, dtype=torch.uint8, device=dev),
        "n_hits": torch.empty(n, dtype=torch.int32, device=dev),
        "barcode": torch.empty((capacity, n), dtype=torch.int64, device=dev),
        "path": torch.empty((capacity, n), **ft),
        "loc0": torch.empty((capacity, n), **ft),
        "loc1": torch.empty((capacity, n), **ft),
        "volume_link": torch.empty((capacity, n), dtype=torch.int16,
                                   device=dev),
    }
    r = abi.ScanResults()
    r.status = out["status"].data_ptr()
    r.n_hits = out["n_hits"].data_ptr()
    r.barcode = out["barcode"].data_ptr()
    r.path = out["path"].data_ptr()
    r.loc[0] = out["loc0"].data_ptr()
    r.loc[1] = out["loc1"].data_ptr()
    r.volume_link = out["volume_link"].data_ptr()
    r.capacity = capacity
    r.precision = 8 if tracks.dtype == torch.float64 else 4
    bb = (C.c_double * 3)(*[float(x) for x in b])
    ts = tracks_struct(tracks)
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    _check(load_library().dprop_helix_scan(
        det.handle, bb, C.byref(ts), n, float(mask_tolerance), C.byref(r),
        C.c_void_p(stream.cuda_stream)))
    out["_inputs"] = tracks
    out["_struct"] = r
    return out


def validate_navigation(scan: dict, results: DeviceResults, max_records: int,
                        path_tolerance: float = 0.1, stream=None):
    """Holes and extra surfaces per track of a propagation (``results`` of
    propagate() with record_all_surfaces = 1) against the helix_scan() of
    the same tracks (dprop_validate_navigation).  Returns the CUDA tensors
    (n_missed, n_extra)."""
    import torch
    n = scan["status"].shape[0]
    dev = scan["status"].device
    missed = torch.empty(n, dtype=torch.int32, device=dev)
    extra = torch.empty(n, dtype=torch.int32, device=dev)
    v = abi.Validation()
    v.n_missed = missed.data_ptr()
    v.n_extra = extra.data_ptr()
    rp = 8 if results.tensors["rec_path"].dtype == torch.float64 else 4
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    _check(load_library().dprop_validate_navigation(
        C.byref(scan["_struct"]), C.byref(results.struct), rp, max_records,
        n, float(path_tolerance), C.byref(v),
        C.c_void_p(stream.cuda_stream)))
    return missed, extra


def alloc_host_results(n: int, max_records: int, pinned: bool = False,
                       with_cov: bool = True,
                       jagged: bool = False) -> tuple[dict, abi.Results]:
    """Host result buffers for propagate_host (float fields as float32).

    jagged=True asks for the records as a jagged array: ``rec_offsets``
    (n + 1 entries) indexes flat record arrays, and only the stored records
    are copied back from the device."""
    if pinned:
        import torch

        def empty(shape, dtype):
            return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()
        import torch as _t
        u8, i32, f32, i64 = _t.uint8, _t.int32, _t.float32, _t.int64
    else:
        def empty(shape, dtype):
            return np.empty(shape, dtype=dtype)
        u8, i32, f32, i64 = np.uint8, np.int32, np.float32, np.int64
    res = {
        "status": empty((n,), u8),
        "n_records": empty((n,), i32),
        "n_steps": empty((n,), i32),
        "n_trials": empty((n,), i32),
        "path_length": empty((n,), f32),
        "final_free": empty((8, n), f32),
        "rec_barcode": empty((max_records, n), i64),
        "rec_bound": empty((6, max_records, n), f32),
        "rec_path": empty((max_records, n), f32),
        "rec_flags": empty((max_records, n), u8),
        "rec_offsets": empty((n + 1,), i64) if jagged else None,
        "n_intersections": empty((n,), i32),
        "n_transports": empty((n,), i32),
        "n_material": empty((n,), i32),
    }
    if with_cov:
        res["rec_cov"] = empty((21, max_records, n), f32)
    r = abi.Results()
    r.status = res["status"].ctypes.data
    r.n_records = res["n_records"].ctypes.data
    r.n_steps = res["n_steps"].ctypes.data
    r.n_trials = res["n_trials"].ctypes.data
    r.path_length = res["path_length"].ctypes.data
    for i in range(8):
        r.final_free[i] = res["final_free"][i].ctypes.data
    r.rec_barcode = res["rec_barcode"].ctypes.data
    for i in range(6):
        r.rec_bound[i] = res["rec_bound"][i].ctypes.data
    if with_cov:
        for i in range(21):
            r.rec_cov[i] = res["rec_cov"][i].ctypes.data
    r.rec_path = res["rec_path"].ctypes.data
    r.rec_flags = res["rec_flags"].ctypes.data
    r.n_intersections = res["n_intersections"].ctypes.data
    r.n_transports = res["n_transports"].ctypes.data
    r.n_material = res["n_material"].ctypes.data
    if jagged:
        r.rec_offsets = res["rec_offsets"].ctypes.data
        # flat views: record j of the jagged array is index j
        for key in ("rec_barcode", "rec_path", "rec_flags"):
            res[key] = res[key].reshape(-1)
        for key in ("rec_bound", "rec_cov"):
            if key in res:
                res[key] = res[key].reshape(res[key].shape[0], -1)
    else:
        del res["rec_offsets"]
    return res, r


def propagate_host(cfg: abi.Config, det: Detector, field: Field,
                   tracks: np.ndarray, launch: abi.Launch | None = None,
                   out: tuple | None = None, jagged: bool = False) -> dict:
    """Propagate host tracks ((8, n) float64); host-to-device copies,
    propagation and device-to-host copies happen inside the call."""
    trk = np.ascontiguousarray(tracks, dtype=np.float64)
    n = trk.shape[1]
    res, r = out if out is not None else alloc_host_results(
        n, cfg.max_records, jagged=jagged)
    ts = tracks_struct(trk)
    lc = launch if launch is not None else make_launch()
    _check(load_library().dprop_propagate_host(
        C.byref(cfg), C.byref(lc), det.handle, field.handle, C.byref(ts),
        C.byref(r), n))
    return res


# the candidates dprop_autotune times, in its order: (method, block_size,
# ctas_per_sm, sort_tracks, steps_per_round, yield_lanes, rounds,
# sort_interval)
AUTOTUNE_CANDIDATES = [
    ("plain", 128, 8, 1, 0, 0, 0, 0), ("plain", 128, 12, 1, 0, 0, 0, 0),
    ("plain", 128, 16, 1, 0, 0, 0, 0), ("plain", 256, 16, 1, 0, 0, 0, 0),
    ("plain", 128, 16, 0, 0, 0, 0, 0),
    ("persistent", 128, 3, 1, 16, 16, 64, 0),
    ("persistent", 128, 3, 1, 16, 16, 64, 1),
    ("persistent", 128, 4, 1, 16, 16, 64, 0),
    ("persistent", 128, 4, 1, 16, 16, 64, 2),
    ("persistent", 128, 5, 1, 16, 16, 64, 0),
    ("persistent", 128, 4, 1, 16, 8, 96, 0),
    ("persistent", 128, 4, 1, 64, 12, 64, 0),
    ("persistent", 128, 4, 0, 16, 16, 64, 0)]


def autotune(cfg: abi.Config, det: Detector, field: Field, tracks,
             use_graph: int = 0, stream=None) -> tuple[abi.Launch, list]:
    """Pick the fastest launch form for these tracks (dprop_autotune)."""
    import torch
    tracks = tracks.contiguous()
    n = tracks.shape[1]
    lc = make_launch(use_graph=use_graph)
    times = (C.c_float * len(AUTOTUNE_CANDIDATES))()
    if stream is None:
        stream = torch.cuda.current_stream(tracks.device)
    ts = tracks_struct(tracks)
    _check(load_library().dprop_autotune(
        C.byref(cfg), det.handle, field.handle, C.byref(ts), n, C.byref(lc),
        times, C.c_void_p(stream.cuda_stream)))
    return lc, list(times)
