// Host-side validation and conversion of dprop_detector_desc into the packed
// device records of tables.cuh.  Every index in the tables is range-checked
// here, before anything is uploaded, so that a kernel can never follow an
// out-of-range link from user input.
#pragma once

#include <string>
#include <vector>

#include "detray_b200/dprop.h"
#include "tables.cuh"

namespace dprop {

template <typename S>
struct host_tables {
    std::vector<dev_volume> volumes;
    std::vector<dev_surface> surfaces;
    std::vector<dev_mask<S>> masks;
    std::vector<dev_transform<S>> transforms;
    std::vector<dev_slab<S>> slabs;
    std::vector<uint32_t> bf_surfaces;
    std::vector<dev_grid<S>> grids;
    std::vector<uint32_t> grid_bins;
    // slab of each volume's homogeneous material (k_invalid: none); empty
    // when no volume carries material
    std::vector<uint32_t> vol_material;

    detector_view<S> view() const { return view_as<true>(); }
    template <bool W>
    detector_view<S, W> view_as() const {
        detector_view<S, W> v;
        v.volumes = volumes.data();
        v.surfaces = surfaces.data();
        v.masks = masks.data();
        v.transforms = transforms.data();
        v.slabs = slabs.data();
        v.bf_surfaces = bf_surfaces.data();
        v.grids = grids.data();
        v.grid_bins = grid_bins.data();
        v.vol_material = vol_material.empty() ? nullptr : vol_material.data();
        v.n_volumes = static_cast<uint32_t>(volumes.size());
        v.n_surfaces = static_cast<uint32_t>(surfaces.size());
        return v;
    }
};

/// Returns an empty string if the tables are consistent, else the problem.
inline std::string validate_desc(const dprop_detector_desc* d) {
    if (!d) {
        return "NULL detector description";
    }
    if (d->abi_version != DPROP_ABI_VERSION) {
        return "ABI version mismatch";
    }
    if (d->n_volumes == 0 || d->n_surfaces == 0) {
        return "empty detector";
    }
    if (!d->volumes || !d->surfaces || !d->masks || !d->transforms ||
        (d->n_slabs && !d->slabs) || (d->n_bf_surfaces && !d->bf_surfaces) ||
        (d->n_grids && !d->grids) || (d->n_grid_bins && !d->grid_bins)) {
        return "NULL table pointer";
    }
    if (d->n_volumes > 0xffffu) {
        return "more than 65535 volumes";
    }
    for (uint32_t i = 0; i < d->n_surfaces; ++i) {
        const dprop_surface_desc& s = d->surfaces[i];
        if (s.mask_end <= s.mask_begin || s.mask_end > d->n_masks ||
            s.mask_end - s.mask_begin > 0xffffu ||
            s.transform >= d->n_transforms || s.volume >= d->n_volumes ||
            s.shape >= DPROP_SHAPE_COUNT || s.kind > DPROP_SF_PASSIVE ||
            s.material_kind > 1u ||
            (s.material != DPROP_INVALID_INDEX && s.material_kind == 0u &&
             s.material >= d->n_slabs) ||
            (s.material != DPROP_INVALID_INDEX && s.material_kind == 1u &&
             (s.material >= d->n_grids ||
              (d->grids[s.material].kind < DPROP_GRID_MATERIAL_CYLINDER ||
               d->grids[s.material].kind > DPROP_GRID_MATERIAL_CARTESIAN)))) {
            return "surface " + std::to_string(i) + " has an out-of-range index";
        }
    }
    for (uint32_t i = 0; i < d->n_masks; ++i) {
        const uint32_t vl = d->masks[i].volume_link;
        if (vl != DPROP_INVALID_LINK && vl >= d->n_volumes) {
            return "mask " + std::to_string(i) + " links to a missing volume";
        }
    }
    for (uint32_t i = 0; i < d->n_volumes; ++i) {
        const dprop_volume_desc& v = d->volumes[i];
        if (v.transform >= d->n_transforms || v.bf_begin > v.bf_end ||
            v.bf_end > d->n_bf_surfaces ||
            (v.grid != DPROP_INVALID_INDEX &&
             (v.grid >= d->n_grids ||
              (d->grids[v.grid].kind != DPROP_GRID_CYLINDER &&
               d->grids[v.grid].kind != DPROP_GRID_DISC)))) {
            return "volume " + std::to_string(i) + " has an out-of-range index";
        }
        if (v.material != DPROP_INVALID_INDEX &&
            (v.material >= d->n_slabs ||
             d->slabs[v.material].kind != DPROP_MATERIAL_SLAB ||
             !(d->slabs[v.material].X0 > 0.) ||
             !(d->slabs[v.material].mean_excitation_energy > 0.))) {
            return "volume " + std::to_string(i) +
                   " has an invalid material index";
        }
    }
    for (uint32_t i = 0; i < d->n_bf_surfaces; ++i) {
        if (d->bf_surfaces[i] >= d->n_surfaces) {
            return "brute-force entry " + std::to_string(i) + " out of range";
        }
    }
    for (uint32_t i = 0; i < d->n_slabs; ++i) {
        if (d->slabs[i].kind > DPROP_MATERIAL_ROD) {
            return "material " + std::to_string(i) + " has an unknown kind";
        }
    }
    // grid_bins entries that are bin ranges of multi-entry grids or slab
    // indices of material maps (the rest are surface indices)
    std::vector<bool> is_range(d->n_grid_bins, false);
    for (uint32_t i = 0; i < d->n_grids; ++i) {
        const dprop_grid_desc& g = d->grids[i];
        const uint64_t nb = static_cast<uint64_t>(g.n_bins[0]) * g.n_bins[1];
        const uint64_t n_entries = nb + (g.multi ? 1u : 0u);
        const bool material_map = g.kind >= DPROP_GRID_MATERIAL_CYLINDER &&
                                  g.kind <= DPROP_GRID_MATERIAL_CARTESIAN;
        if ((g.kind != DPROP_GRID_CYLINDER && g.kind != DPROP_GRID_DISC &&
             !material_map) ||
            g.n_bins[0] == 0 || g.n_bins[1] == 0 || g.multi > 1u ||
            (material_map && g.multi != 0u) ||
            static_cast<uint64_t>(g.bin_offset) + n_entries > d->n_grid_bins ||
            g.transform >= d->n_transforms ||
            !(g.axis_max[0] > g.axis_min[0]) || !(g.axis_max[1] > g.axis_min[1])) {
            return "grid " + std::to_string(i) + " is inconsistent";
        }
        if (material_map) {
            // bins hold slab indices
            for (uint64_t b = 0; b < nb; ++b) {
                const uint64_t e = g.bin_offset + b;
                is_range[e] = true;
                if (d->grid_bins[e] >= d->n_slabs ||
                    d->slabs[d->grid_bins[e]].kind != DPROP_MATERIAL_SLAB) {
                    return "material map " + std::to_string(i) +
                           " has a bin without a slab";
                }
            }
        }
        if (g.multi) {
            for (uint64_t b = 0; b < n_entries; ++b) {
                const uint64_t e = g.bin_offset + b;
                is_range[e] = true;
                if (d->grid_bins[e] > d->n_grid_bins ||
                    (b > 0 && d->grid_bins[e] < d->grid_bins[e - 1])) {
                    return "grid " + std::to_string(i) +
                           " has an inconsistent bin range";
                }
            }
        }
    }
    for (uint32_t i = 0; i < d->n_grid_bins; ++i) {
        if (!is_range[i] && d->grid_bins[i] != DPROP_INVALID_INDEX &&
            d->grid_bins[i] >= d->n_surfaces) {
            return "grid bin " + std::to_string(i) + " out of range";
        }
    }
    return {};
}

// One material slab descriptor -> the device slab.
template <typename S>
dev_slab<S> convert_slab(const dprop_slab_desc& s) {
    dev_slab<S> o{};
    o.thickness = static_cast<S>(s.thickness);
    o.thickness_in_X0 = static_cast<S>(s.thickness_in_X0);
    o.molar_electron_density = static_cast<S>(s.molar_electron_density);
    o.mean_excitation_energy = static_cast<S>(s.mean_excitation_energy);
    o.density_a = static_cast<S>(s.density_a);
    o.density_m = static_cast<S>(s.density_m);
    o.density_x0 = static_cast<S>(s.density_x0);
    o.density_x1 = static_cast<S>(s.density_x1);
    o.density_c = static_cast<S>(s.density_c);
    o.has_density_effect = s.has_density_effect ? S(1) : S(0);
    o.X0 = static_cast<S>(s.X0);
    o.is_rod = (s.kind == DPROP_MATERIAL_ROD) ? S(1) : S(0);
    return o;
}

template <typename S>
host_tables<S> convert_desc(const dprop_detector_desc* d) {
    host_tables<S> t;
    t.volumes.resize(d->n_volumes);
    for (uint32_t i = 0; i < d->n_volumes; ++i) {
        t.volumes[i] = dev_volume{d->volumes[i].transform, d->volumes[i].bf_begin,
                                  d->volumes[i].bf_end, d->volumes[i].grid};
    }
    t.surfaces.resize(d->n_surfaces);
    for (uint32_t i = 0; i < d->n_surfaces; ++i) {
        const dprop_surface_desc& s = d->surfaces[i];
        dev_surface o{};
        o.barcode = s.barcode;
        o.transform = s.transform;
        o.material = s.material;
        o.mask_begin = s.mask_begin;
        o.n_masks = static_cast<uint16_t>(s.mask_end - s.mask_begin);
        o.shape = s.shape;
        o.kind = s.kind;
        o.volume = s.volume;
        o.material_map = s.material_kind;
        t.surfaces[i] = o;
    }
    t.masks.resize(d->n_masks);
    for (uint32_t i = 0; i < d->n_masks; ++i) {
        dev_mask<S> m{};
        for (int k = 0; k < 6; ++k) {
            m.v[k] = static_cast<S>(d->masks[i].values[k]);
        }
        m.volume_link = d->masks[i].volume_link;
        t.masks[i] = m;
    }
    t.transforms.resize(d->n_transforms);
    for (uint32_t i = 0; i < d->n_transforms; ++i) {
        const dprop_transform_desc& tr = d->transforms[i];
        dev_transform<S> o{};
        for (int k = 0; k < 9; ++k) {
            o.rot[k] = static_cast<S>(tr.rot[k]);
            o.inv_rot[k] = static_cast<S>(tr.inv_rot[k]);
        }
        for (int k = 0; k < 3; ++k) {
            o.t[k] = static_cast<S>(tr.translation[k]);
            o.inv_t[k] = static_cast<S>(tr.inv_translation[k]);
        }
        t.transforms[i] = o;
    }
    t.slabs.resize(d->n_slabs);
    for (uint32_t i = 0; i < d->n_slabs; ++i) {
        t.slabs[i] = convert_slab<S>(d->slabs[i]);
    }
    t.bf_surfaces.assign(d->bf_surfaces, d->bf_surfaces + d->n_bf_surfaces);
    t.grids.resize(d->n_grids);
    for (uint32_t i = 0; i < d->n_grids; ++i) {
        const dprop_grid_desc& g = d->grids[i];
        dev_grid<S> o{};
        o.kind = g.kind;
        o.n0 = g.n_bins[0];
        o.n1 = g.n_bins[1];
        o.bin_offset = g.bin_offset;
        o.transform = g.transform;
        o.multi = g.multi;
        o.min0 = static_cast<S>(g.axis_min[0]);
        o.max0 = static_cast<S>(g.axis_max[0]);
        o.min1 = static_cast<S>(g.axis_min[1]);
        o.max1 = static_cast<S>(g.axis_max[1]);
        o.radius = static_cast<S>(g.radius);
        t.grids[i] = o;
    }
    t.grid_bins.assign(d->grid_bins, d->grid_bins + d->n_grid_bins);
    bool any_material = false;
    for (uint32_t i = 0; i < d->n_volumes; ++i) {
        any_material = any_material ||
                       d->volumes[i].material != DPROP_INVALID_INDEX;
    }
    if (any_material) {
        t.vol_material.resize(d->n_volumes);
        for (uint32_t i = 0; i < d->n_volumes; ++i) {
            t.vol_material[i] = d->volumes[i].material;
        }
    }
    return t;
}

// True if any volume carries homogeneous material (the stepper then
// evaluates the energy loss dq/p/ds: the full kernel variant).
inline bool has_volume_material(const dprop_detector_desc* d) {
    for (uint32_t i = 0; i < d->n_volumes; ++i) {
        if (d->volumes[i].material != DPROP_INVALID_INDEX) {
            return true;
        }
    }
    return false;
}

}  // namespace dprop
