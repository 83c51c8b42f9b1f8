"""ctypes mirror of the C ABI declared in include/detray_b200/dprop.h.

The structures here must match the header field by field; a CPU test
compiles the header and compares every struct size and field offset.  This
module only describes the boundary - it does not load anything by itself.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

DPROP_ABI_VERSION = 3
DPROP_INVALID_INDEX = 0xFFFFFFFF
DPROP_INVALID_LINK = 0xFFFF

# dprop_status
DPROP_OK = 0
DPROP_E_INVALID = 1
DPROP_E_CUDA = 2
DPROP_E_NO_DEVICE = 3
DPROP_E_OOM = 4
DPROP_E_TIMEOUT = 5
DPROP_E_UNSUPPORTED = 6

# dprop_track_status
TRK_EXITED = 0
TRK_PATH_LIMIT = 1
TRK_STALLED = 2
TRK_NO_SURFACE = 3
TRK_MAX_ITER = 4
TRK_NOT_RUN = 5
TRK_NONFINITE = 6

# dprop_shape
SHAPE_RECTANGLE = 0
SHAPE_TRAPEZOID = 1
SHAPE_RING = 2
SHAPE_CYLINDER = 3
SHAPE_CONCENTRIC_CYL = 4
SHAPE_LINE = 5

# dprop_surface_kind
SF_PORTAL = 0
SF_SENSITIVE = 1
SF_PASSIVE = 2

# dprop_material_kind
MATERIAL_SLAB = 0
MATERIAL_ROD = 1

# dprop_grid_kind
GRID_NONE = 0
GRID_CYLINDER = 1
GRID_DISC = 2
GRID_MATERIAL_CYLINDER = 3
GRID_MATERIAL_DISC = 4
GRID_MATERIAL_CARTESIAN = 5

# dprop_method
METHOD_PLAIN = 0
METHOD_PERSISTENT = 1

# record flags
REC_TRANSPORTED = 1
REC_PORTAL = 2
REC_MATERIAL = 4


class SurfaceDesc(C.Structure):
    _fields_ = [
        ("barcode", C.c_uint64),
        ("mask_begin", C.c_uint32),
        ("mask_end", C.c_uint32),
        ("transform", C.c_uint32),
        ("material", C.c_uint32),
        ("volume", C.c_uint32),
        ("shape", C.c_uint8),
        ("kind", C.c_uint8),
        ("material_kind", C.c_uint8),
        ("pad", C.c_uint8),
    ]


class MaskDesc(C.Structure):
    _fields_ = [
        ("values", C.c_double * 6),
        ("volume_link", C.c_uint32),
        ("pad", C.c_uint32),
    ]


class TransformDesc(C.Structure):
    _fields_ = [
        ("rot", C.c_double * 9),
        ("translation", C.c_double * 3),
        ("inv_rot", C.c_double * 9),
        ("inv_translation", C.c_double * 3),
    ]


class SlabDesc(C.Structure):
    _fields_ = [
        ("thickness", C.c_double),
        ("thickness_in_X0", C.c_double),
        ("X0", C.c_double),
        ("molar_electron_density", C.c_double),
        ("mean_excitation_energy", C.c_double),
        ("density_a", C.c_double),
        ("density_m", C.c_double),
        ("density_x0", C.c_double),
        ("density_x1", C.c_double),
        ("density_c", C.c_double),
        ("has_density_effect", C.c_uint32),
        ("kind", C.c_uint32),
    ]


class GridDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32),
        ("n_bins", C.c_uint32 * 2),
        ("bin_offset", C.c_uint32),
        ("transform", C.c_uint32),
        ("multi", C.c_uint32),
        ("axis_min", C.c_double * 2),
        ("axis_max", C.c_double * 2),
        ("radius", C.c_double),
    ]


class VolumeDesc(C.Structure):
    _fields_ = [
        ("transform", C.c_uint32),
        ("bf_begin", C.c_uint32),
        ("bf_end", C.c_uint32),
        ("grid", C.c_uint32),
        ("material", C.c_uint32),
    ]


class DetectorDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("n_volumes", C.c_uint32),
        ("n_surfaces", C.c_uint32),
        ("n_masks", C.c_uint32),
        ("n_transforms", C.c_uint32),
        ("n_slabs", C.c_uint32),
        ("n_bf_surfaces", C.c_uint32),
        ("n_grids", C.c_uint32),
        ("n_grid_bins", C.c_uint32),
        ("volumes", C.POINTER(VolumeDesc)),
        ("surfaces", C.POINTER(SurfaceDesc)),
        ("masks", C.POINTER(MaskDesc)),
        ("transforms", C.POINTER(TransformDesc)),
        ("slabs", C.POINTER(SlabDesc)),
        ("bf_surfaces", C.POINTER(C.c_uint32)),
        ("grids", C.POINTER(GridDesc)),
        ("grid_bins", C.POINTER(C.c_uint32)),
    ]


class Config(C.Structure):
    _fields_ = [
        ("min_stepsize", C.c_float),
        ("rk_error_tol", C.c_float),
        ("step_constraint", C.c_float),
        ("path_limit", C.c_float),
        ("max_rk_updates", C.c_uint32),
        ("use_mean_loss", C.c_uint8),
        ("use_eloss_gradient", C.c_uint8),
        ("use_field_gradient", C.c_uint8),
        ("do_covariance_transport", C.c_uint8),
        ("min_mask_tolerance", C.c_float),
        ("max_mask_tolerance", C.c_float),
        ("mask_tolerance_scalor", C.c_float),
        ("path_tolerance", C.c_float),
        ("overstep_tolerance", C.c_float),
        ("search_window", C.c_uint32 * 2),
        ("accumulated_error", C.c_float),
        ("n_scattering_stddev", C.c_int32),
        ("estimate_scattering_noise", C.c_uint8),
        ("use_path_limit_aborter", C.c_uint8),
        ("use_material_interactor", C.c_uint8),
        ("record_all_surfaces", C.c_uint8),
        ("mass", C.c_float),
        ("pdg", C.c_int32),
        ("max_records", C.c_uint32),
        ("max_iterations", C.c_uint32),
    ]


class Tracks(C.Structure):
    _fields_ = [
        ("pos", C.c_void_p * 3),
        ("time", C.c_void_p),
        ("dir", C.c_void_p * 3),
        ("qop", C.c_void_p),
    ]


class Sequence(C.Structure):
    """dprop_sequence: surface sequences for dprop_propagate_direct."""
    _fields_ = [
        ("barcodes", C.c_void_p),
        ("length", C.c_void_p),
        ("max_length", C.c_uint32),
        ("direction", C.c_int32),
        ("start_barcode", C.c_void_p),
        ("start_bound", C.c_void_p * 6),
    ]


# dprop_scan_status
SCAN_OK = 0
SCAN_OVERFLOW = 1
SCAN_EMPTY = 2


class ScanResults(C.Structure):
    """dprop_scan_results: output of dprop_helix_scan."""
    _fields_ = [
        ("status", C.c_void_p),
        ("n_hits", C.c_void_p),
        ("barcode", C.c_void_p),
        ("path", C.c_void_p),
        ("loc", C.c_void_p * 2),
        ("volume_link", C.c_void_p),
        ("capacity", C.c_uint32),
        ("precision", C.c_uint32),
    ]


class Validation(C.Structure):
    """dprop_validation: output of dprop_validate_navigation."""
    _fields_ = [
        ("n_missed", C.c_void_p),
        ("n_extra", C.c_void_p),
    ]


class Results(C.Structure):
    _fields_ = [
        ("status", C.c_void_p),
        ("n_records", C.c_void_p),
        ("n_steps", C.c_void_p),
        ("n_trials", C.c_void_p),
        ("path_length", C.c_void_p),
        ("final_free", C.c_void_p * 8),
        ("rec_barcode", C.c_void_p),
        ("rec_bound", C.c_void_p * 6),
        ("rec_cov", C.c_void_p * 21),
        ("rec_path", C.c_void_p),
        ("rec_flags", C.c_void_p),
        ("n_intersections", C.c_void_p),
        ("n_transports", C.c_void_p),
        ("n_material", C.c_void_p),
        ("rec_offsets", C.c_void_p),
    ]


class Launch(C.Structure):
    _fields_ = [
        ("method", C.c_uint32),
        ("block_size", C.c_uint32),
        ("ctas_per_sm", C.c_uint32),
        ("sort_tracks", C.c_uint32),
        ("use_graph", C.c_uint32),
        ("precision", C.c_uint32),
        ("steps_per_round", C.c_uint32),
        ("rounds", C.c_uint32),
        ("yield_lanes", C.c_uint32),
        ("sort_interval", C.c_uint32),
        ("tail_tracks", C.c_uint32),
        ("reserved", C.c_uint32 * 1),
    ]


# Adjoint-mode tape sizes in floats (dprop.h DPROP_TAPE_*_FLOATS)
TAPE_RECORD_FLOATS = 27
TAPE_TRACK_FLOATS = 35


class Tape(C.Structure):
    _fields_ = [
        ("rec", C.c_void_p),
        ("init", C.c_void_p),
    ]


class Gradients(C.Structure):
    _fields_ = [
        ("grad_bound", C.c_void_p * 6),
        ("grad_free", C.c_void_p * 8),
        ("grad_align", C.c_void_p),
    ]


def default_config_values() -> dict:
    """The reference defaults (stepping_config.hpp:27-77,
    navigation_config.hpp:23-56, intersection_config.hpp:20-33) plus the
    actor-chain switches; same values as dprop_config_default()."""
    flt_max = 3.4028234663852886e38
    return dict(
        min_stepsize=1e-4,
        rk_error_tol=1e-4,
        step_constraint=flt_max,
        path_limit=5000.0,
        max_rk_updates=10000,
        use_mean_loss=1,
        use_eloss_gradient=0,
        use_field_gradient=0,
        do_covariance_transport=1,
        min_mask_tolerance=1e-5,
        max_mask_tolerance=3.0,
        mask_tolerance_scalor=5e-2,
        path_tolerance=1e-3,
        overstep_tolerance=-1.0,
        search_window=(0, 0),
        accumulated_error=0.001,
        n_scattering_stddev=3,
        estimate_scattering_noise=1,
        use_path_limit_aborter=1,
        use_material_interactor=1,
        record_all_surfaces=0,
        # the reference's muon mass, a float product
        # (definitions/pdg_particle.hpp:84: 105.6583755f * unit<float>::MeV)
        mass=float(np.float32(np.float32(105.6583755) * np.float32(1e-3))),
        pdg=13,
        max_records=32,
        max_iterations=200000,
    )


def make_config(**overrides) -> Config:
    vals = default_config_values()
    unknown = set(overrides) - set(vals)
    if unknown:
        raise KeyError(f"unknown dprop_config fields: {sorted(unknown)}")
    vals.update(overrides)
    cfg = Config()
    for k, v in vals.items():
        if k == "search_window":
            cfg.search_window[0] = int(v[0])
            cfg.search_window[1] = int(v[1])
        else:
            setattr(cfg, k, v)
    return cfg
