// Device layout of the detector tables and the magnetic field.
//
// The host hands over dprop_detector_desc (double precision, C structs); the
// library converts it once into the packed records below and keeps them in
// HBM for the lifetime of the detector.  They replace the six stores of
// detray::detector (core/include/detray/core/detector.hpp:101-167):
// volumes, surfaces, transforms, masks, materials and accelerators.  The whole
// toy detector is ~0.6 MB, i.e. L2-resident; records are sized in 16/32-byte
// multiples so that one lookup touches one or two 32-byte sectors.
#pragma once

#include "defs.cuh"

namespace dprop {

constexpr uint32_t k_invalid = 0xffffffffu;
constexpr uint32_t k_invalid_link = 0xffffu;

enum shape_id : uint8_t {
    e_rectangle = 0,
    e_trapezoid = 1,
    e_ring = 2,
    e_cylinder = 3,
    e_concentric_cylinder = 4,
    e_line = 5,
};

enum surface_kind : uint8_t { e_portal = 0, e_sensitive = 1, e_passive = 2 };

// 32 bytes.  barcode = geometry::identifier value (identifier.hpp:153-157).
struct alignas(16) dev_surface {
    uint64_t barcode;
    uint32_t transform;
    uint32_t material;   // slab index or k_invalid
    uint32_t mask_begin;
    uint16_t n_masks;
    uint8_t shape;
    uint8_t kind;
    uint32_t volume;
    uint32_t material_map;  // 1: material indexes a material-map grid
};

// 32 bytes (fp32) / 64 bytes (fp64): bounds + next-volume link.
template <typename S>
struct alignas(16) dev_mask {
    S v[6];
    uint32_t volume_link;
    uint32_t pad;
};

// Placement and its inverse, as stored by detray's transform3
// (algebra/generic/impl/generic_transform3.hpp): rotation columns x, y, z and
// the translation, then the same for the inverse.
template <typename S>
struct alignas(16) dev_transform {
    S rot[9];  // column-major: rot[3 * c + r]
    S t[3];
    S inv_rot[9];
    S inv_t[3];

    DPROP_HD vec3<S> x() const { return {rot[0], rot[1], rot[2]}; }
    DPROP_HD vec3<S> y() const { return {rot[3], rot[4], rot[5]}; }
    DPROP_HD vec3<S> z() const { return {rot[6], rot[7], rot[8]}; }
    DPROP_HD vec3<S> translation() const { return {t[0], t[1], t[2]}; }

    // transform3::point_to_local / point_to_global
    DPROP_HD vec3<S> point_to_local(vec3<S> p) const {
        return {inv_rot[0] * p.x + inv_rot[3] * p.y + inv_rot[6] * p.z + inv_t[0],
                inv_rot[1] * p.x + inv_rot[4] * p.y + inv_rot[7] * p.z + inv_t[1],
                inv_rot[2] * p.x + inv_rot[5] * p.y + inv_rot[8] * p.z + inv_t[2]};
    }
    DPROP_HD vec3<S> point_to_global(vec3<S> p) const {
        return {rot[0] * p.x + rot[3] * p.y + rot[6] * p.z + t[0],
                rot[1] * p.x + rot[4] * p.y + rot[7] * p.z + t[1],
                rot[2] * p.x + rot[5] * p.y + rot[8] * p.z + t[2]};
    }
    DPROP_HD vec3<S> vector_to_local(vec3<S> v) const {
        return {inv_rot[0] * v.x + inv_rot[3] * v.y + inv_rot[6] * v.z,
                inv_rot[1] * v.x + inv_rot[4] * v.y + inv_rot[7] * v.z,
                inv_rot[2] * v.x + inv_rot[5] * v.y + inv_rot[8] * v.z};
    }
};

// Homogeneous material slab with the quantities the interaction formulas
// read (material_slab.hpp, material.hpp).
template <typename S>
struct alignas(16) dev_slab {
    S thickness;
    S thickness_in_X0;
    S molar_electron_density;
    S mean_excitation_energy;
    S density_a, density_m, density_x0, density_x1, density_c;
    S has_density_effect;  // 0 or 1
    S X0;                  // radiation length
    S is_rod;              // 0: slab of thickness t; 1: rod of radius t
};

struct alignas(16) dev_volume {
    uint32_t transform;
    uint32_t bf_begin;
    uint32_t bf_end;
    uint32_t grid;
};

template <typename S>
struct alignas(16) dev_grid {
    uint32_t kind;  // 1 cylinder (phi, z), 2 disc (r, phi); material maps:
                    // 3 cylinder (phi, z), 4 disc (r, phi)
    uint32_t n0, n1;
    uint32_t bin_offset;
    uint32_t transform;
    uint32_t multi;  // 1: bins hold [begin, end) ranges into grid_bins
    uint32_t pad[2];
    S min0, max0, min1, max1;
    S radius;
    S pad2[3];
};

// Read-only view handed to the kernels by value.  W = false promises that the
// detector holds no line surfaces, material rods, multi-entry grid bins,
// material maps or volume material: the code for them is then left out of
// the propagation.
template <typename S, bool W = true>
struct detector_view {
    const dev_volume* volumes;
    const dev_surface* surfaces;
    const dev_mask<S>* masks;
    const dev_transform<S>* transforms;
    const dev_slab<S>* slabs;
    const uint32_t* bf_surfaces;
    const dev_grid<S>* grids;
    const uint32_t* grid_bins;
    const uint32_t* vol_material;  // [n_volumes] slab of the volume's
                                   // material or k_invalid; NULL: none has
    uint32_t n_volumes;
    uint32_t n_surfaces;

    // The homogeneous material of volume v, or NULL.
    DPROP_HD const dev_slab<S>* volume_material(uint32_t v) const {
        if constexpr (W) {
            if (vol_material != nullptr) {
                const uint32_t m = vol_material[v];
                return m != k_invalid ? slabs + m : nullptr;
            }
        }
        return nullptr;
    }
};

// Magnetic field view.  kind 0: constant; kind 1: (r, phi, z) node map of
// float4 (B_r, B_phi, B_z, 0), node index (iz * n_phi + iphi) * n_r + ir.
template <typename S>
struct field_view {
    uint32_t kind;
    uint32_t n_r, n_phi, n_z;
    S b[3];
    S r_lo, r_step_inv;
    S phi_lo, phi_step_inv;
    S z_lo, z_step_inv;
    const float4* nodes;
};

}  // namespace dprop
