"""ORACLE - test infrastructure only.

Python access to the reference detray propagator compiled by
``oracle/ref/Makefile`` into ``oracle/_ref/libdetray_ref_{f64,f32}.so``.
Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product never does.

Functions:
  * ``build_toy`` / ``build_telescope``: the reference's detector builders
    (tests/include/detray/test/common/build_toy_detector.hpp:1237,
    build_telescope_detector.hpp:187) and their flattened tables;
  * ``propagate``: propagator::propagate over a batch with OpenMP
    (core/include/detray/propagator/propagator.hpp:260-400), actor chain
    pathlimit_aborter -> parameter_updater<pointwise_material_interactor>
    -> surface recorder, results in the dprop_results layout (doubles).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from detray_b200 import abi

_HERE = Path(__file__).resolve().parent
REF_DIR = _HERE / "_ref"


class _RefTelCfg(C.Structure):
    _fields_ = [
        ("half_x", C.c_double),
        ("half_y", C.c_double),
        ("positions", C.POINTER(C.c_double)),
        ("n_positions", C.c_uint32),
        ("volume_material", C.c_uint32),
        ("pilot_dir", C.c_double * 3),
        ("mat_thickness", C.c_double),
        ("envelope", C.c_double),
    ]


class _RefToyCfg(C.Structure):
    _fields_ = [
        ("n_brl_layers", C.c_uint32),
        ("n_edc_layers", C.c_uint32),
        ("module_mat_thickness", C.c_double),
        ("beampipe_mat_thickness", C.c_double),
        ("use_material_maps", C.c_uint32),
        ("pad", C.c_uint32),
    ]


class RefFieldDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32),
        ("n", C.c_uint32 * 3),
        ("b", C.c_double * 3),
        ("lo", C.c_double * 3),
        ("hi", C.c_double * 3),
        ("values", C.POINTER(C.c_float)),
    ]


_LIBS: dict[str, C.CDLL] = {}


def available(precision: str = "f64") -> bool:
    return (REF_DIR / f"libdetray_ref_{precision}.so").exists()


def load(precision: str = "f64") -> C.CDLL:
    if precision in _LIBS:
        return _LIBS[precision]
    path = REF_DIR / f"libdetray_ref_{precision}.so"
    if not path.exists():
        raise FileNotFoundError(
            f"{path} missing: build it with `make -C oracle/ref` "
            "(needs the reference checkout)")
    lib = C.CDLL(str(path))
    lib.ref_last_error.restype = C.c_char_p
    lib.ref_build_toy.argtypes = [C.POINTER(_RefToyCfg), C.POINTER(C.c_void_p)]
    lib.ref_build_telescope.argtypes = [C.POINTER(_RefTelCfg),
                                        C.POINTER(C.c_void_p)]
    lib.ref_tables.argtypes = [C.c_void_p, C.POINTER(abi.DetectorDesc)]
    lib.ref_destroy.argtypes = [C.c_void_p]
    lib.ref_propagate.argtypes = [
        C.c_void_p, C.POINTER(RefFieldDesc), C.POINTER(abi.Config),
        C.POINTER(C.c_void_p), C.c_uint64, C.POINTER(abi.Results), C.c_int,
        C.c_int, C.c_int]
    lib.ref_propagate_jac.argtypes = [
        C.c_void_p, C.POINTER(RefFieldDesc), C.POINTER(abi.Config),
        C.POINTER(C.c_void_p), C.c_uint64, C.POINTER(abi.Results), C.c_int,
        C.c_int, C.c_int, C.c_void_p]
    lib.ref_material_slab.argtypes = [C.c_char_p, C.c_double,
                                      C.POINTER(abi.SlabDesc),
                                      C.POINTER(C.c_double)]
    lib.ref_bethe.argtypes = [C.c_char_p, C.c_int, C.c_double,
                              C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.ref_field_eval.argtypes = [C.POINTER(RefFieldDesc),
                                   C.POINTER(C.c_double), C.c_uint64,
                                   C.POINTER(C.c_double)]
    _optional_argtypes(lib)
    _LIBS[precision] = lib
    return lib


def _optional_argtypes(lib) -> None:
    """Entry points that a library built by an older recipe may lack."""
    if not hasattr(lib, "ref_propagate_direct"):
        return
    lib.ref_propagate_direct.argtypes = [
        C.c_void_p, C.POINTER(RefFieldDesc), C.POINTER(abi.Config),
        C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int,
        C.c_void_p, C.c_void_p, C.POINTER(abi.Results), C.c_int]
    if hasattr(lib, "ref_helix_scan"):
        lib.ref_helix_scan.argtypes = [
            C.c_void_p, C.POINTER(C.c_double), C.c_void_p, C.c_uint64,
            C.c_double, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]


class RefDetector:
    """A reference-built detector plus its flattened tables."""

    def __init__(self, lib: C.CDLL, handle: C.c_void_p):
        self._lib = lib
        self.handle = handle
        self.desc = abi.DetectorDesc()
        lib.ref_tables(handle, C.byref(self.desc))

    def __del__(self):
        if getattr(self, "handle", None):
            self._lib.ref_destroy(self.handle)
            self.handle = None

    def tables(self) -> dict:
        """Copies of the flat tables as numpy structured arrays."""
        d = self.desc

        def arr(ptr, n, ctype):
            if n == 0:
                return np.zeros(0, dtype=np.ctypeslib.as_ctypes_type(ctype)
                                if False else None)
            buf = (ctype * n).from_address(C.addressof(ptr.contents))
            return np.ctypeslib.as_array(buf).copy()

        out = {}
        out["volumes"] = np.ctypeslib.as_array(
            (abi.VolumeDesc * d.n_volumes).from_address(
                C.addressof(d.volumes.contents))).copy()
        out["surfaces"] = np.ctypeslib.as_array(
            (abi.SurfaceDesc * d.n_surfaces).from_address(
                C.addressof(d.surfaces.contents))).copy()
        out["masks"] = np.ctypeslib.as_array(
            (abi.MaskDesc * d.n_masks).from_address(
                C.addressof(d.masks.contents))).copy()
        out["transforms"] = np.ctypeslib.as_array(
            (abi.TransformDesc * d.n_transforms).from_address(
                C.addressof(d.transforms.contents))).copy()
        if d.n_slabs:
            out["slabs"] = np.ctypeslib.as_array(
                (abi.SlabDesc * d.n_slabs).from_address(
                    C.addressof(d.slabs.contents))).copy()
        else:
            out["slabs"] = np.zeros(0, dtype=np.dtype(abi.SlabDesc))
        out["bf_surfaces"] = np.ctypeslib.as_array(
            (C.c_uint32 * d.n_bf_surfaces).from_address(
                C.addressof(d.bf_surfaces.contents))).copy()
        if d.n_grids:
            out["grids"] = np.ctypeslib.as_array(
                (abi.GridDesc * d.n_grids).from_address(
                    C.addressof(d.grids.contents))).copy()
            out["grid_bins"] = np.ctypeslib.as_array(
                (C.c_uint32 * d.n_grid_bins).from_address(
                    C.addressof(d.grid_bins.contents))).copy()
        else:
            out["grids"] = np.zeros(0, dtype=np.dtype(abi.GridDesc))
            out["grid_bins"] = np.zeros(0, dtype=np.uint32)
        return out


def _check(lib, rc):
    if rc != 0:
        raise RuntimeError(lib.ref_last_error().decode())


def build_toy(n_brl_layers=4, n_edc_layers=7, module_mat_thickness=0.15,
              beampipe_mat_thickness=0.0, use_material_maps=False,
              precision="f64") -> RefDetector:
    lib = load(precision)
    cfg = _RefToyCfg(n_brl_layers, n_edc_layers, module_mat_thickness,
                     beampipe_mat_thickness, int(use_material_maps), 0)
    h = C.c_void_p()
    _check(lib, lib.ref_build_toy(C.byref(cfg), C.byref(h)))
    return RefDetector(lib, h)


class _RefWireCfg(C.Structure):
    _fields_ = [
        ("n_layers", C.c_uint32),
        ("square_cells", C.c_uint32),
        ("first_layer_inner_radius", C.c_double),
        ("half_z", C.c_double),
        ("cell_size", C.c_double),
        ("stereo_angle", C.c_double),
        ("mat_radius", C.c_double),
    ]


def build_wire_chamber(n_layers=10, square_cells=True,
                       first_layer_inner_radius=500.0, half_z=1000.0,
                       cell_size=10.0, stereo_angle=0.05, mat_radius=0.015,
                       precision="f64") -> RefDetector:
    """The reference's wire chamber (tests/include/detray/test/common/
    build_wire_chamber.hpp) with drift cells (square) or straw tubes."""
    lib = load(precision)
    lib.ref_build_wire_chamber.argtypes = [C.POINTER(_RefWireCfg),
                                           C.POINTER(C.c_void_p)]
    cfg = _RefWireCfg(n_layers, int(square_cells), first_layer_inner_radius,
                      half_z, cell_size, stereo_angle, mat_radius)
    h = C.c_void_p()
    _check(lib, lib.ref_build_wire_chamber(C.byref(cfg), C.byref(h)))
    return RefDetector(lib, h)


# homogeneous volume materials of build_telescope(volume_material=...)
VOLUME_MATERIALS = {None: 0, "cesium_iodide": 1, "iron": 2,
                    "argon_liquid": 3, "silicon": 4}


def build_telescope(positions=tuple(50.0 * i for i in range(10)),
                    half_x=500.0, half_y=500.0, pilot_dir=(1.0, 0.0, 0.0),
                    mat_thickness=0.3, envelope=0.0, volume_material=None,
                    precision="f64") -> RefDetector:
    """The reference's telescope (build_telescope_detector.hpp:187), with
    an optional homogeneous volume material filling the telescope volume
    (tel_det_config::volume_material)."""
    lib = load(precision)
    pos = (C.c_double * len(positions))(*positions)
    cfg = _RefTelCfg(half_x, half_y, pos, len(positions),
                     VOLUME_MATERIALS[volume_material],
                     (C.c_double * 3)(*pilot_dir), mat_thickness, envelope)
    h = C.c_void_p()
    _check(lib, lib.ref_build_telescope(C.byref(cfg), C.byref(h)))
    return RefDetector(lib, h)


def field_desc(field) -> tuple[RefFieldDesc, object]:
    """Translate a detray_b200 field specification (dict) into the oracle's
    descriptor.  Returns (desc, keepalive)."""
    fd = RefFieldDesc()
    keep = None
    if field["kind"] == "const":
        fd.kind = 0
        for i in range(3):
            fd.b[i] = float(field["b"][i])
    else:
        fd.kind = 1
        vals = np.ascontiguousarray(field["values"], dtype=np.float32)
        keep = vals
        for i in range(3):
            fd.n[i] = int(field["n"][i])
            fd.lo[i] = float(field["lo"][i])
            fd.hi[i] = float(field["hi"][i])
        fd.values = vals.ctypes.data_as(C.POINTER(C.c_float))
    return fd, keep


def field_eval(field, xyz: np.ndarray, precision="f64") -> np.ndarray:
    lib = load(precision)
    fd, keep = field_desc(field)
    pts = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    out = np.zeros_like(pts)
    lib.ref_field_eval(C.byref(fd), pts.ctypes.data_as(C.POINTER(C.c_double)),
                       pts.shape[0], out.ctypes.data_as(C.POINTER(C.c_double)))
    del keep
    return out


def alloc_results(n: int, max_records: int) -> tuple[dict, abi.Results]:
    """Host result buffers (doubles for floating fields) + the ABI struct."""
    res = {
        "status": np.full(n, 255, dtype=np.uint8),
        "n_records": np.zeros(n, dtype=np.uint32),
        "n_steps": np.zeros(n, dtype=np.uint32),
        "n_trials": np.zeros(n, dtype=np.uint32),
        "path_length": np.zeros(n, dtype=np.float64),
        "final_free": np.zeros((8, n), dtype=np.float64),
        "rec_barcode": np.full((max_records, n), np.iinfo(np.uint64).max,
                               dtype=np.uint64),
        "rec_bound": np.zeros((6, max_records, n), dtype=np.float64),
        "rec_cov": np.zeros((21, max_records, n), dtype=np.float64),
        "rec_path": np.zeros((max_records, n), dtype=np.float64),
        "rec_flags": np.zeros((max_records, n), dtype=np.uint8),
        "n_intersections": np.zeros(n, dtype=np.uint32),
        "n_transports": np.zeros(n, dtype=np.uint32),
        "n_material": np.zeros(n, dtype=np.uint32),
    }
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
    for i in range(21):
        r.rec_cov[i] = res["rec_cov"][i].ctypes.data
    r.rec_path = res["rec_path"].ctypes.data
    r.rec_flags = res["rec_flags"].ctypes.data
    r.n_intersections = res["n_intersections"].ctypes.data
    r.n_transports = res["n_transports"].ctypes.data
    r.n_material = res["n_material"].ctypes.data
    return res, r


def propagate(det: RefDetector, field: dict, cfg: abi.Config,
              tracks: np.ndarray, n_threads: int = 0, chunk: int = 1,
              abort_reasons: bool = True, full_jacobian: bool = False) -> dict:
    """Run the reference propagator on ``tracks`` (shape (8, n) float64, the
    free vector rows [x, y, z, t, tx, ty, tz, q/p]).  With ``full_jacobian``
    the result also holds "rec_jac" [36][max_records][n]: the reference's
    accumulated full Jacobian (row-major 6 x 6) after each transported
    record."""
    lib = det._lib
    trk = np.ascontiguousarray(tracks, dtype=np.float64)
    n = trk.shape[1]
    ptrs = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    res, r = alloc_results(n, cfg.max_records)
    fd, keep = field_desc(field)
    if n_threads <= 0:
        n_threads = os.cpu_count() or 1
    jac = None
    if full_jacobian:
        jac = np.zeros((36, cfg.max_records, n), dtype=np.float64)
        res["rec_jac"] = jac
    _check(lib, lib.ref_propagate_jac(
        det.handle, C.byref(fd), C.byref(cfg), ptrs, n, C.byref(r), n_threads,
        chunk, int(abort_reasons),
        jac.ctypes.data_as(C.c_void_p) if jac is not None else None))
    del keep
    return res


def propagate_direct(det: RefDetector, field: dict, cfg: abi.Config,
                     sequence: np.ndarray, lengths: np.ndarray,
                     direction: int = 1, tracks: np.ndarray | None = None,
                     start_barcode: np.ndarray | None = None,
                     start_bound: np.ndarray | None = None,
                     n_threads: int = 0) -> dict:
    """The reference's propagation with the direct navigator along the
    surface sequences ``sequence`` (barcodes, shape (max_length, n)) of
    ``lengths`` entries, forward (+1) or backward (-1); starting from the
    free ``tracks`` (8, n) or from bound parameters ``start_bound`` (6, n)
    on the surfaces ``start_barcode`` (n)."""
    lib = det._lib
    seq = np.ascontiguousarray(sequence, dtype=np.uint64)
    lens = np.ascontiguousarray(lengths, dtype=np.uint32)
    n = lens.shape[0]
    max_len = seq.shape[0]
    keep = []
    trk_ptrs = None
    if tracks is not None:
        trk = np.ascontiguousarray(tracks, dtype=np.float64)
        keep.append(trk)
        trk_ptrs = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    sb_ptrs = None
    sbc = None
    if start_barcode is not None:
        sbc = np.ascontiguousarray(start_barcode, dtype=np.uint64)
        sb = np.ascontiguousarray(start_bound, dtype=np.float64)
        keep.append(sb)
        sb_ptrs = (C.c_void_p * 6)(*[sb[i].ctypes.data for i in range(6)])
    res, r = alloc_results(n, cfg.max_records)
    fd, fkeep = field_desc(field)
    if n_threads <= 0:
        n_threads = os.cpu_count() or 1
    _check(lib, lib.ref_propagate_direct(
        det.handle, C.byref(fd), C.byref(cfg),
        C.cast(trk_ptrs, C.c_void_p) if trk_ptrs is not None else None, n,
        seq.ctypes.data if max_len > 0 else None, lens.ctypes.data, max_len,
        int(direction), sbc.ctypes.data if sbc is not None else None,
        C.cast(sb_ptrs, C.c_void_p) if sb_ptrs is not None else None,
        C.byref(r), n_threads))
    del fkeep, keep
    return res


def alloc_scan(n: int, capacity: int) -> dict:
    """Host arrays for a helix scan (oracle, host core)."""
    return {
        "status": np.full(n, 255, dtype=np.uint8),
        "n_hits": np.zeros(n, dtype=np.uint32),
        "barcode": np.zeros((capacity, n), dtype=np.uint64),
        "path": np.zeros((capacity, n), dtype=np.float64),
        "loc0": np.zeros((capacity, n), dtype=np.float64),
        "loc1": np.zeros((capacity, n), dtype=np.float64),
        "volume_link": np.zeros((capacity, n), dtype=np.uint16),
    }


def scan_pointers(res: dict) -> list:
    return [res[k].ctypes.data for k in ("status", "n_hits", "barcode",
                                         "path", "loc0", "loc1",
                                         "volume_link")]


def helix_scan(det: RefDetector, b, tracks: np.ndarray, mask_tol: float,
               capacity: int = 256, n_threads: int = 0) -> dict:
    """The reference's navigation-validation helix scan of ``tracks``
    ((8, n) float64) in the constant field ``b``: per track the
    intersections with all surfaces along the helix, sorted by path and cut
    after the first world exit (slot-major, ``capacity`` slots)."""
    lib = det._lib
    trk = np.ascontiguousarray(tracks, dtype=np.float64)
    n = trk.shape[1]
    ptrs = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    bb = (C.c_double * 3)(*b)
    res = alloc_scan(n, capacity)
    if n_threads <= 0:
        n_threads = os.cpu_count() or 1
    _check(lib, lib.ref_helix_scan(det.handle, bb, C.cast(ptrs, C.c_void_p),
                                   n, mask_tol, capacity,
                                   *scan_pointers(res), n_threads))
    return res


def material_slab(name: str, thickness: float, precision="f64"):
    """(slab descriptor, mass density) of a predefined reference material."""
    lib = load(precision)
    d = abi.SlabDesc()
    rho = C.c_double()
    _check(lib, lib.ref_material_slab(name.encode(), thickness, C.byref(d),
                                      C.byref(rho)))
    return d, rho.value


def bethe(name: str, pdg: int, p: float, precision="f64"):
    """The reference's mean stopping power (detray units) and its q/p
    derivative for a particle of momentum p in a predefined material."""
    lib = load(precision)
    v = C.c_double()
    dv = C.c_double()
    _check(lib, lib.ref_bethe(name.encode(), pdg, p, C.byref(v), C.byref(dv)))
    return v.value, dv.value


def gpu_available() -> bool:
    """The reference's CUDA propagation kernel, built for sm_100a."""
    return (REF_DIR / "libdetray_ref_gpu.so").exists()


def gpu_toy_bench(cfg: abi.Config, bz: float, tracks: np.ndarray,
                  warmup: int = 3, steps: int = 10) -> dict:
    """Time the reference's own CUDA propagation kernel
    (propagator_benchmark_kernel of its CUDA benchmark, rebuilt for sm_100a;
    oracle/ref/ref_gpu*.{cu,cpp}) on ``tracks`` through the toy detector in
    a constant field bz along z.  Returns ms per launch and the number of
    tracks whose propagate() returned true."""
    lib = C.CDLL(str(REF_DIR / "libdetray_ref_gpu.so"))
    lib.refgpu_last_error.restype = C.c_char_p
    lib.refgpu_toy_bench.argtypes = [
        C.POINTER(abi.Config), C.c_double, C.POINTER(C.c_void_p), C.c_uint64,
        C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
    trk = np.ascontiguousarray(tracks, dtype=np.float64)
    ptrs = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    ms = C.c_double()
    ok = C.c_uint64()
    rc = lib.refgpu_toy_bench(C.byref(cfg), bz, ptrs, trk.shape[1], warmup,
                              steps, C.byref(ms), C.byref(ok))
    if rc != 0:
        raise RuntimeError(lib.refgpu_last_error().decode())
    return {"ms_per_step": ms.value, "n_exited": int(ok.value)}


def gpu_toy_map_bench(cfg: abi.Config, fmap: dict, tracks: np.ndarray,
                      warmup: int = 2, steps: int = 5) -> dict:
    """Time the reference tutorial's CUDA propagation kernel (path-limit
    aborter and parameter updater with the material interactor, built per
    thread as in tutorials/src/device/cuda/propagation_kernel.cu; oracle/ref/
    ref_gpu*.{cu,cpp}) on ``tracks`` through the toy detector in the field
    map ``fmap`` (detray_b200.fields format).  Returns ms per launch and the
    number of tracks whose propagate() returned true."""
    lib = C.CDLL(str(REF_DIR / "libdetray_ref_gpu.so"))
    lib.refgpu_last_error.restype = C.c_char_p
    lib.refgpu_toy_map_bench.argtypes = [
        C.POINTER(abi.Config), C.POINTER(C.c_double), C.POINTER(C.c_double),
        C.POINTER(C.c_uint32), C.c_void_p, C.POINTER(C.c_void_p), C.c_uint64,
        C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
    trk = np.ascontiguousarray(tracks, dtype=np.float64)
    ptrs = (C.c_void_p * 8)(*[trk[i].ctypes.data for i in range(8)])
    lo = (C.c_double * 3)(*fmap["lo"])
    hi = (C.c_double * 3)(*fmap["hi"])
    nn = (C.c_uint32 * 3)(*fmap["n"])
    vals = np.ascontiguousarray(fmap["values"], dtype=np.float32)
    ms = C.c_double()
    ok = C.c_uint64()
    rc = lib.refgpu_toy_map_bench(C.byref(cfg), lo, hi, nn,
                                  vals.ctypes.data_as(C.c_void_p), ptrs,
                                  trk.shape[1], warmup, steps, C.byref(ms),
                                  C.byref(ok))
    if rc != 0:
        raise RuntimeError(lib.refgpu_last_error().decode())
    return {"ms_per_step": ms.value, "n_exited": int(ok.value)}


def json_available() -> bool:
    """The reference's JSON detector writer and reader (oracle/ref/
    ref_json.cpp, built when nlohmann/json is found)."""
    return (REF_DIR / "ref_json").exists()


def write_json(kind: str, directory) -> list:
    """Build a benchmark detector with the reference's builders and write it
    with detray::io::write_detector into ``directory``.  kind: toy,
    toy_maps, telescope, wire_cells, wire_straws.  Returns the written
    .json files (those with data)."""
    import subprocess
    from pathlib import Path
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    subprocess.run([str(REF_DIR / "ref_json"), "write", kind, str(d)],
                   check=True, capture_output=True)
    return sorted(str(p) for p in d.glob("*.json"))


def read_json_tables(kind: str, files, out_path) -> dict:
    """Read detray JSON files with the reference's reader
    (detray::io::read_detector into the detector type of ``kind``) and
    return dprop::flatten of the result as table arrays."""
    import subprocess
    from detray_b200 import geometry
    subprocess.run([str(REF_DIR / "ref_json"), "read", kind, str(out_path),
                    *[str(f) for f in files]], check=True, capture_output=True)
    return geometry.read_raw_tables(out_path)
