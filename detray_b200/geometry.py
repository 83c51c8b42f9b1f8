"""Flat detector tables on the host: file I/O and the C-ABI descriptor.

A detector reaches the device as the flat tables of ``dprop_detector_desc``
(include/detray_b200/dprop.h), the flattened form of detray's detector stores
(core/include/detray/core/detector.hpp:57-355).  This module keeps those
tables as numpy structured arrays, reads/writes them, and builds the ctypes
descriptor that ``dprop_detector_create`` consumes.

Benchmark geometries ship as ``detray_b200/geometries/*.npz``; they are the
reference's own toy and telescope builders flattened by the product adapter
(see oracle/geometries/make_geometries.py).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import abi

GEOMETRY_DIR = Path(__file__).resolve().parent / "geometries"

TABLES = [
    ("volumes", abi.VolumeDesc),
    ("surfaces", abi.SurfaceDesc),
    ("masks", abi.MaskDesc),
    ("transforms", abi.TransformDesc),
    ("slabs", abi.SlabDesc),
    ("bf_surfaces", C.c_uint32),
    ("grids", abi.GridDesc),
    ("grid_bins", C.c_uint32),
]


def dtype_of(ctype) -> np.dtype:
    return np.dtype(ctype)


def read_raw_tables(path) -> dict:
    """Read the raw table file written by oracle/geometries/export_geometry.cpp
    (the geometry regeneration step)."""
    data = Path(path).read_bytes()
    header = np.frombuffer(data[:48], dtype=np.uint32)
    if header[0] != 0x4F454744:
        raise ValueError(f"{path}: not a detray-b200 table file")
    if header[1] != abi.DPROP_ABI_VERSION:
        raise ValueError(f"{path}: table ABI version {header[1]}")
    counts = header[2:10]
    off = 48
    out = {}
    for (name, ctype), n in zip(TABLES, counts):
        dt = dtype_of(ctype)
        nbytes = int(n) * dt.itemsize
        out[name] = np.frombuffer(data[off:off + nbytes], dtype=dt).copy()
        off += nbytes
    if off != len(data):
        raise ValueError(f"{path}: trailing bytes in table file")
    return out


def write_raw_tables(tables: dict, path) -> None:
    """Write tables (as load_geometry returns them) to a raw table file, the
    form read_raw_tables and the C++ dprop::read_raw_tables read."""
    header = np.zeros(12, np.uint32)
    header[0] = 0x4F454744
    header[1] = abi.DPROP_ABI_VERSION
    parts = []
    for i, (name, ctype) in enumerate(TABLES):
        arr = np.ascontiguousarray(tables[name], dtype=dtype_of(ctype))
        header[2 + i] = arr.shape[0]
        parts.append(arr.tobytes())
    Path(path).write_bytes(header.tobytes() + b"".join(parts))


def save_npz(tables: dict, path) -> None:
    np.savez_compressed(path, **{k: tables[k] for k, _ in TABLES})


def load_npz(path) -> dict:
    with np.load(path) as z:
        out = {}
        for name, ctype in TABLES:
            arr = np.ascontiguousarray(z[name])
            dt = dtype_of(ctype)
            if name == "volumes" and arr.dtype.names is not None and \
                    "material" not in arr.dtype.names:
                # tables written before volumes carried a material index
                vol = np.zeros(arr.shape[0], dtype=dt)
                for f in arr.dtype.names:
                    vol[f] = arr[f]
                vol["material"] = abi.DPROP_INVALID_INDEX
                out[name] = vol
                continue
            out[name] = arr.view(dt).reshape(-1)
        return out


def load_geometry(name: str) -> dict:
    """One of the committed benchmark geometries by name."""
    return load_npz(GEOMETRY_DIR / f"{name}.npz")


class Descriptor:
    """A dprop_detector_desc pointing into numpy tables kept alive here."""

    def __init__(self, tables: dict):
        self.tables = {name: np.ascontiguousarray(tables[name],
                                                  dtype=dtype_of(ctype))
                       for name, ctype in TABLES}
        d = abi.DetectorDesc()
        d.abi_version = abi.DPROP_ABI_VERSION
        t = self.tables
        d.n_volumes = len(t["volumes"])
        d.n_surfaces = len(t["surfaces"])
        d.n_masks = len(t["masks"])
        d.n_transforms = len(t["transforms"])
        d.n_slabs = len(t["slabs"])
        d.n_bf_surfaces = len(t["bf_surfaces"])
        d.n_grids = len(t["grids"])
        d.n_grid_bins = len(t["grid_bins"])

        def ptr(name, ctype):
            arr = t[name]
            if arr.size == 0:
                return C.cast(None, C.POINTER(ctype))
            return arr.ctypes.data_as(C.POINTER(ctype))

        d.volumes = ptr("volumes", abi.VolumeDesc)
        d.surfaces = ptr("surfaces", abi.SurfaceDesc)
        d.masks = ptr("masks", abi.MaskDesc)
        d.transforms = ptr("transforms", abi.TransformDesc)
        d.slabs = ptr("slabs", abi.SlabDesc)
        d.bf_surfaces = ptr("bf_surfaces", C.c_uint32)
        d.grids = ptr("grids", abi.GridDesc)
        d.grid_bins = ptr("grid_bins", C.c_uint32)
        self.desc = d


def decode_barcode(bc) -> dict:
    """Fields of a detray geometry::identifier (identifier.hpp:153-157)."""
    bc = np.asarray(bc, dtype=np.uint64)
    return {
        "volume": (bc >> np.uint64(52)) & np.uint64(0xFFF),
        "id": (bc >> np.uint64(48)) & np.uint64(0xF),
        "index": (bc >> np.uint64(27)) & np.uint64(0x1FFFFF),
        "transform": (bc >> np.uint64(6)) & np.uint64(0x1FFFFF),
        "extra": bc & np.uint64(0x3F),
    }
