"""Detector JSON reader: detray's JSON geometry files -> the flat tables of
the C ABI (dprop_detector_desc), ready for ``propagator.Detector``.

This is the product-side counterpart of ``detray::io::read_detector``
(io/include/detray/io/frontend/detector_reader.hpp:62-103) followed by
``dprop::flatten`` (include/detray_b200/detray_adapter.hpp): it reads the
files the reference's ``write_detector`` produces (or ACTS exports in the
same format) without a C++ detray build, and lays the tables out exactly as
the reference's reader + builders + flatten would:

* geometry (tag "geometry", io/include/detray/io/json/detail/
  json_geometry_io.hpp): volumes in file order; per volume the placement
  transform first, then the surfaces grouped as the geometry reader feeds its
  surface factories (io/include/detray/io/backend/geometry_reader.hpp:87-170):
  portals before the other surfaces, each group ordered by IO shape id and
  kept in file order inside a shape, every surface (and its transform) put at
  its ``index_in_coll`` when the file gives one
  (builders/surface_factory.hpp:185-245, surface_factory_interface.hpp:
  158-176); cylinder surfaces become concentric portal cylinders with their
  z shift folded into the mask bounds (geometry_reader.hpp:215-232);
  surface indices and transform indices become global by the volume's
  offsets (builders/volume_builder.hpp:105-305);
* homogeneous material (tag "homogeneous_material", json_material_io.hpp;
  backend/homogeneous_material_reader.hpp:45-150): slabs and rods built as
  ``material(X0, L0, Ar, Z, mass_rho, state)`` (material/material.hpp:42-53,
  molar density from mass density and Ar, mean excitation energy
  16 eV * Z^0.9 since files carry no density-effect data);
* material maps (tag "material_maps", backend/material_map_reader.hpp:45-
  170): one slab per bin, unlisted bins empty;
* surface grids (tag "surface_grids", json_grids_io.hpp; backend/detail/
  grid_reader.hpp): bins hold volume-local surface indices
  (builders/grid_builder.hpp:173-230); a cylinder grid's reference radius is
  the mean of the smallest and largest portal-cylinder radius of its volume
  (grid_builder.hpp:232-272); a volume with a grid keeps only its portals and
  passives in the brute-force list (volume_builder.hpp:266-296).

Transform inverses are computed as R^T and -R^T t of the rigid placement;
the reference inverts the 4x4 matrix numerically, the two agree to a few
ulp.  Unsupported content (annulus or 3D shapes, volume material, more than
one surface grid per volume) raises ``ValueError``.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from detray_b200 import abi, geometry
from detray_b200.units import g as _gram

# io::shape_id (io/include/detray/io/frontend/definitions.hpp:25-41)
_IO_CYLINDER2 = 2
_IO_PORTAL_CYLINDER2 = 4
_IO_SHAPES = {
    _IO_PORTAL_CYLINDER2: abi.SHAPE_CONCENTRIC_CYL,
    5: abi.SHAPE_RECTANGLE,
    6: abi.SHAPE_RING,
    7: abi.SHAPE_TRAPEZOID,
    8: abi.SHAPE_LINE,  # drift_cell (square cross section)
    9: abi.SHAPE_LINE,  # straw_tube (circular cross section)
}
_IO_DRIFT_CELL = 8

# io::material_id (definitions.hpp:48-63)
_IO_SLAB = 6
_IO_ROD = 7

# io::accel_id (definitions.hpp:72-82)
_IO_POLAR2_GRID = 3
_IO_CONCENTRIC_CYL2_GRID = 4

# geometry::identifier bit layout (geometry/identifier.hpp:153-157)
_EXTRA_INVALID = 0x3F

_EV = 1e-9  # GeV
_SURFACE_PORTAL = 0
_SURFACE_SENSITIVE = 1
_SURFACE_PASSIVE = 2


def _load(path) -> dict:
    with open(path, "rb") as f:
        return json.load(f)


def _data(doc: dict) -> dict:
    # a writer with nothing to write leaves "data" null
    return doc.get("data") or {}


def _tag(doc: dict) -> str:
    return doc["header"]["common"]["tag"]


def _transform(payload: dict) -> np.void:
    """transform3(t, x, y, z) from a transform payload
    (geometry_reader.hpp:175-197): the rotation array holds the x, y and z
    axes one after the other, i.e. the rotation matrix column-major."""
    t = np.asarray(payload["translation"], dtype=np.float64)
    rot = np.asarray(payload["rotation"], dtype=np.float64)
    return _make_transform(t, rot)


def _make_transform(t: np.ndarray, rot: np.ndarray) -> np.void:
    d = np.zeros(1, dtype=geometry.dtype_of(abi.TransformDesc))[0]
    d["rot"][:] = rot
    d["translation"][:] = t
    r = rot.reshape(3, 3)  # row k = axis k = column k of R
    # inverse rotation R^T: its column k is row k of R
    d["inv_rot"][:] = r.T.reshape(9)
    d["inv_translation"][:] = -(r @ t)
    return d


_IDENTITY = np.array([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0])


def _slab(entry: dict) -> np.void:
    """material_slab / material_rod from a surface material payload
    (homogeneous_material_reader.hpp:123-150, material/material.hpp,
    material/material_slab.hpp:33-38)."""
    x0, _l0, ar, z, mass_rho, _molar_rho, _state = (
        float(v) for v in entry["material"]["params"])
    thickness = float(entry["thickness"])
    d = np.zeros(1, dtype=geometry.dtype_of(abi.SlabDesc))[0]
    molar_rho = 0.0 if mass_rho == 0.0 else mass_rho / (ar * _gram / 1.0)
    d["thickness"] = thickness
    d["thickness_in_X0"] = thickness / x0
    d["X0"] = x0
    d["molar_electron_density"] = z * molar_rho
    d["mean_excitation_energy"] = 16.0 * _EV * z ** 0.9
    d["has_density_effect"] = 0
    mtype = int(entry["type"])
    if mtype == _IO_ROD:
        d["kind"] = abi.MATERIAL_ROD
    elif mtype == _IO_SLAB:
        d["kind"] = abi.MATERIAL_SLAB
    else:
        raise ValueError(f"unsupported homogeneous material type {mtype}")
    return d


class _Surface:
    __slots__ = ("kind", "shape", "io_shape", "masks", "trf", "local_trf")

    def __init__(self, sf: dict):
        masks = sf.get("masks")
        if masks is None:
            masks = [sf["mask"]]
        if not masks:
            raise ValueError("surface payload without masks")
        io_shape = int(masks[0]["shape"])
        if io_shape == _IO_CYLINDER2:
            io_shape = _IO_PORTAL_CYLINDER2
        if io_shape not in _IO_SHAPES:
            raise ValueError(f"mask shape id {io_shape} is not on the "
                             "propagation path")
        self.io_shape = io_shape
        self.shape = _IO_SHAPES[io_shape]
        self.kind = int(sf["type"])
        trf = sf["transform"]
        t = np.asarray(trf["translation"], dtype=np.float64)
        rot = np.asarray(trf["rotation"], dtype=np.float64)
        self.masks = []
        if io_shape == _IO_PORTAL_CYLINDER2:
            # fold the z shift into the bounds, identity placement
            z_shift = t[2]
            for m in masks:
                b = [float(v) for v in m["boundaries"]]
                b[1] += z_shift
                b[2] += z_shift
                self.masks.append((b, int(m["volume_link"])))
            self.trf = _make_transform(np.zeros(3), _IDENTITY)
        else:
            for m in masks:
                b = [float(v) for v in m["boundaries"]]
                if self.shape == abi.SHAPE_LINE:
                    b = b[:2] + [1.0 if io_shape == _IO_DRIFT_CELL else 0.0]
                self.masks.append((b, int(m["volume_link"])))
            self.trf = _make_transform(t, rot)


def _place(container: list, value, index):
    """surface_factory_interface::insert_in_container: push back without a
    position, else resize and put at the position."""
    if index is None:
        container.append(value)
        return len(container) - 1
    if len(container) < index + 1:
        container.extend([None] * (index + 1 - len(container)))
    container[index] = value
    return index


def _read_volume(vol: dict) -> list:
    """Volume-local surface list in the order the volume builder stores it."""
    portal_groups: dict[int, list] = {}
    other_groups: dict[int, list] = {}
    for sf in vol["surfaces"]:
        s = _Surface(sf)
        groups = portal_groups if s.kind == _SURFACE_PORTAL else other_groups
        groups.setdefault(s.io_shape, []).append(
            (s, sf.get("index_in_coll")))
    surfaces: list = []
    transforms: list = []
    for groups in (portal_groups, other_groups):
        for key in sorted(groups):
            for s, idx in groups[key]:
                idx = None if idx is None else int(idx)
                s.local_trf = _place(transforms, s.trf, idx)
                _place(surfaces, s, idx)
    if any(s is None for s in surfaces) or any(t is None for t in transforms):
        raise ValueError(f"volume {vol.get('name')}: surface indices in the "
                         "file leave holes")
    return surfaces, transforms


def _axes(grid: dict) -> tuple[list, list, list]:
    n, lo, hi = [], [], []
    for ax in grid["axes"]:
        if int(ax.get("binning", 0)) != 0:
            raise ValueError("only regular grid axes are supported")
        edges = [float(e) for e in ax["edges"]]
        n.append(int(ax["bins"]))
        lo.append(edges[0])
        hi.append(edges[-1])
    if len(n) != 2:
        raise ValueError("only 2D grids are supported")
    return n, lo, hi


def read_detector(files) -> dict:
    """Read detray JSON detector files (any order; the kind of each file is
    taken from its header tag) into the flat C-ABI tables.

    Returns the dict of numpy structured arrays ``propagator.Detector``
    takes (same layout as ``geometry.load_geometry``)."""
    docs: dict[str, dict] = {}
    for f in files:
        doc = _load(Path(f))
        tag = _tag(doc)
        if tag in docs:
            raise ValueError(f"two files with tag {tag!r}")
        if tag not in ("geometry", "homogeneous_material", "material_maps",
                       "surface_grids"):
            raise ValueError(f"unsupported file tag {tag!r} in {f}")
        docs[tag] = doc
    if "geometry" not in docs:
        raise ValueError("no geometry file given")

    # ---------------------------------------------------------- geometry
    volumes_in = _data(docs["geometry"]).get("volumes", [])
    vol_surfaces = []     # per volume: local surface list
    vol_trf_index = []    # per volume: index of its placement transform
    vol_sf_offset = []    # per volume: global index of its first surface
    transforms = []
    n_surfaces = 0
    for v in volumes_in:
        vol_trf_index.append(len(transforms))
        transforms.append(_transform(v["transform"]))
        surfaces, local_trfs = _read_volume(v)
        trf_offset = len(transforms)
        transforms.extend(local_trfs)
        for s in surfaces:
            s.local_trf += trf_offset
        vol_sf_offset.append(n_surfaces)
        n_surfaces += len(surfaces)
        vol_surfaces.append(surfaces)
    n_vol = len(volumes_in)

    # ------------------------------------------------- material per surface
    material: dict[tuple[int, int], tuple[str, object]] = {}
    if "homogeneous_material" in docs:
        for mv in _data(docs["homogeneous_material"]).get("volumes", []):
            vi = int(mv["volume_link"])
            entries = mv.get("surface_material", mv.get("material_slabs", []))
            for e in entries:
                material[(vi, int(e["surface_idx"]))] = ("slab", _slab(e))
    if "material_maps" in docs:
        for gv in _data(docs["material_maps"]).get("grids", []):
            vi = int(gv["volume_link"])
            for gd in gv["grid_data"]:
                key = (vi, int(gd["owner_link"]))
                if key in material:
                    raise ValueError(f"surface {key} has two materials")
                material[key] = ("map", gd)
    nav_grids: dict[int, dict] = {}
    if "surface_grids" in docs:
        for gv in _data(docs["surface_grids"]).get("grids", []):
            vi = int(gv["volume_link"])
            for gd in gv["grid_data"]:
                if int(gd["owner_link"]) != vi:
                    raise ValueError("grid owner differs from its volume")
                if vi in nav_grids:
                    raise ValueError(f"volume {vi}: more than one surface "
                                     "grid")
                nav_grids[vi] = gd
    for (vi, li) in material:
        if vi >= n_vol or li >= len(vol_surfaces[vi]):
            raise ValueError(f"material for missing surface {(vi, li)}")

    # ---------------------------------------------------------- flatten
    surf_t = geometry.dtype_of(abi.SurfaceDesc)
    mask_t = geometry.dtype_of(abi.MaskDesc)
    slab_t = geometry.dtype_of(abi.SlabDesc)
    grid_t = geometry.dtype_of(abi.GridDesc)
    vol_t = geometry.dtype_of(abi.VolumeDesc)
    surfaces_out = np.zeros(n_surfaces, dtype=surf_t)
    masks_out = []
    slabs_out = []
    grids_out = []
    grid_bins: list[int] = []
    for vi, surfaces in enumerate(vol_surfaces):
        for li, s in enumerate(surfaces):
            gi = vol_sf_offset[vi] + li
            o = surfaces_out[gi]
            o["barcode"] = ((vi << 52) | (s.kind << 48) | (gi << 27)
                            | (s.local_trf << 6) | _EXTRA_INVALID)
            o["transform"] = s.local_trf
            o["volume"] = vi
            o["shape"] = s.shape
            o["kind"] = s.kind
            o["mask_begin"] = len(masks_out)
            for bounds, link in s.masks:
                md = np.zeros(1, dtype=mask_t)[0]
                md["values"][:len(bounds)] = bounds[:6]
                md["volume_link"] = (abi.DPROP_INVALID_LINK
                                     if link >= 0xFFFF else link)
                masks_out.append(md)
            o["mask_end"] = len(masks_out)
            o["material"] = abi.DPROP_INVALID_INDEX
            mat = material.get((vi, li))
            if mat is None:
                continue
            kind, payload = mat
            if kind == "slab":
                o["material"] = len(slabs_out)
                slabs_out.append(payload)
                continue
            gd = np.zeros(1, dtype=grid_t)[0]
            if s.shape == abi.SHAPE_CONCENTRIC_CYL:
                gd["kind"] = abi.GRID_MATERIAL_CYLINDER
            elif s.shape == abi.SHAPE_RING:
                gd["kind"] = abi.GRID_MATERIAL_DISC
            elif s.shape in (abi.SHAPE_RECTANGLE, abi.SHAPE_TRAPEZOID):
                gd["kind"] = abi.GRID_MATERIAL_CARTESIAN
            else:
                raise ValueError("material map on a line surface")
            n, lo, hi = _axes(payload)
            gd["n_bins"][:] = n
            gd["axis_min"][:] = lo
            gd["axis_max"][:] = hi
            gd["transform"] = s.local_trf
            gd["bin_offset"] = len(grid_bins)
            nb = n[0] * n[1]
            bin_slab = [None] * nb
            for b in payload["bins"]:
                b0, b1 = (int(x) for x in b["loc_index"])
                if not (0 <= b0 < n[0] and 0 <= b1 < n[1]):
                    raise ValueError("material map bin out of range")
                for c in b["content"]:
                    bin_slab[b0 + b1 * n[0]] = _slab(c)
            for sl in bin_slab:
                grid_bins.append(len(slabs_out))
                slabs_out.append(sl if sl is not None
                                 else np.zeros(1, dtype=slab_t)[0])
            o["material"] = len(grids_out)
            o["material_kind"] = 1
            grids_out.append(gd)

    volumes_out = np.zeros(n_vol, dtype=vol_t)
    bf_out: list[int] = []
    for vi, surfaces in enumerate(vol_surfaces):
        vo = volumes_out[vi]
        vo["transform"] = vol_trf_index[vi]
        vo["grid"] = abi.DPROP_INVALID_INDEX
        vo["material"] = abi.DPROP_INVALID_INDEX
        off = vol_sf_offset[vi]
        has_grid = vi in nav_grids
        vo["bf_begin"] = len(bf_out)
        for li, s in enumerate(surfaces):
            if not (has_grid and s.kind == _SURFACE_SENSITIVE):
                bf_out.append(off + li)
        vo["bf_end"] = len(bf_out)
        if not has_grid:
            continue
        gd_in = nav_grids[vi]
        acc = int(gd_in["grid_link"]["type"])
        gd = np.zeros(1, dtype=grid_t)[0]
        if acc == _IO_CONCENTRIC_CYL2_GRID:
            gd["kind"] = abi.GRID_CYLINDER
            radii = [s.masks[0][0][0] for s in surfaces
                     if s.kind == _SURFACE_PORTAL
                     and s.shape == abi.SHAPE_CONCENTRIC_CYL]
            gd["radius"] = (0.5 * (min(radii) + max(radii))) if radii else 0.0
        elif acc == _IO_POLAR2_GRID:
            gd["kind"] = abi.GRID_DISC
        else:
            raise ValueError(f"surface grid type {acc} is not supported")
        n, lo, hi = _axes(gd_in)
        gd["n_bins"][:] = n
        gd["axis_min"][:] = lo
        gd["axis_max"][:] = hi
        gd["transform"] = vol_trf_index[vi]
        gd["bin_offset"] = len(grid_bins)
        nb = n[0] * n[1]
        content: list[list[int]] = [[] for _ in range(nb)]
        for b in gd_in["bins"]:
            b0, b1 = (int(x) for x in b["loc_index"])
            if not (0 <= b0 < n[0] and 0 <= b1 < n[1]):
                raise ValueError("surface grid bin out of range")
            for c in b["content"]:
                c = int(c)
                if c >= 0xFFFFFFFF:
                    continue
                if c >= len(surfaces):
                    raise ValueError("surface grid entry out of range")
                content[b0 + b1 * n[0]].append(off + c)
        if max((len(c) for c in content), default=0) <= 1:
            gd["multi"] = 0
            for c in content:
                grid_bins.append(c[0] if c else abi.DPROP_INVALID_INDEX)
        else:
            gd["multi"] = 1
            pos = len(grid_bins) + nb + 1
            for c in content:
                grid_bins.append(pos)
                pos += len(c)
            grid_bins.append(pos)
            for c in content:
                grid_bins.extend(c)
        vo["grid"] = len(grids_out)
        grids_out.append(gd)

    def arr(items, dt):
        return (np.array(items, dtype=dt) if items
                else np.zeros(0, dtype=dt))

    return {
        "volumes": volumes_out,
        "surfaces": surfaces_out,
        "masks": arr(masks_out, mask_t),
        "transforms": arr(transforms, geometry.dtype_of(abi.TransformDesc)),
        "slabs": arr(slabs_out, slab_t),
        "bf_surfaces": np.asarray(bf_out, dtype=np.uint32),
        "grids": arr(grids_out, grid_t),
        "grid_bins": np.asarray(grid_bins, dtype=np.uint32),
    }
