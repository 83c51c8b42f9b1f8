/*
 * Host-side C++ adapter for code that already holds a detray detector.
 *
 * dprop::flatten(det) turns a detray::detector<metadata, host containers>
 * (core/include/detray/core/detector.hpp:57-355) into the flat tables of
 * dprop_detector_desc, which dprop_detector_create() uploads.  It plays the
 * role of detray::get_buffer(det, mr, copy) + get_data(buffer)
 * (core/include/detray/core/detail/container_buffers.hpp:82-195): one call
 * per detector, after which the device copy is immutable.
 *
 * The adapter is header-only and generic over the detector metadata: masks,
 * materials and accelerators are reached through detray's own store visitors
 * (core/include/detray/core/detail/multi_store.hpp), so the toy, telescope and
 * wire-chamber metadata work unchanged.  It needs the detray headers on the
 * include path; the product library itself does not.
 */
#pragma once

#include "detray_b200/dprop.h"
#include "detray_b200/flat_tables.hpp"

#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace dprop {

namespace adapter_detail {

template <typename shape_t>
constexpr int shape_code() {
    if constexpr (std::is_same_v<shape_t, detray::rectangle2D>) {
        return DPROP_SHAPE_RECTANGLE;
    } else if constexpr (std::is_same_v<shape_t, detray::trapezoid2D>) {
        return DPROP_SHAPE_TRAPEZOID;
    } else if constexpr (std::is_same_v<shape_t, detray::ring2D>) {
        return DPROP_SHAPE_RING;
    } else if constexpr (std::is_same_v<shape_t, detray::cylinder2D>) {
        return DPROP_SHAPE_CYLINDER;
    } else if constexpr (std::is_same_v<shape_t,
                                        detray::concentric_cylinder2D>) {
        return DPROP_SHAPE_CONCENTRIC_CYL;
    } else if constexpr (std::is_same_v<shape_t, detray::line<true>> ||
                         std::is_same_v<shape_t, detray::line<false>>) {
        return DPROP_SHAPE_LINE;
    } else {
        return -1;
    }
}

/// Mask-store visitor: appends every mask of one surface.
struct mask_copier {
    template <typename mask_group_t, typename range_t>
    void operator()(const mask_group_t& group, const range_t& range,
                    flat_detector& out, dprop_surface_desc& sf) const {
        using mask_t = typename mask_group_t::value_type;
        using shape_t = typename mask_t::shape;
        constexpr int code = shape_code<shape_t>();
        if constexpr (code < 0) {
            throw std::runtime_error("dprop::flatten: mask shape " +
                                     std::string(shape_t::name) +
                                     " is not on the propagation path");
        } else {
            std::size_t lo{0u};
            std::size_t hi{0u};
            if constexpr (detray::concepts::interval<range_t>) {
                lo = range.lower();
                hi = range.upper();
            } else {
                lo = range;
                hi = range + 1u;
            }
            sf.mask_begin = static_cast<uint32_t>(out.masks.size());
            for (std::size_t i = lo; i < hi; ++i) {
                const auto& m = group[i];
                dprop_mask_desc md{};
                const auto& v = m.values();
                for (std::size_t k = 0; k < v.size() && k < 6u; ++k) {
                    md.values[k] = static_cast<double>(v[k]);
                }
                if constexpr (code == DPROP_SHAPE_LINE) {
                    md.values[2] = shape_t::square_cross_sect ? 1.0 : 0.0;
                }
                const auto vl = m.volume_link();
                md.volume_link =
                    (vl == std::numeric_limits<std::decay_t<decltype(vl)>>::max())
                        ? DPROP_INVALID_LINK
                        : static_cast<uint32_t>(vl);
                out.masks.push_back(md);
            }
            sf.mask_end = static_cast<uint32_t>(out.masks.size());
            sf.shape = static_cast<uint8_t>(code);
        }
    }
};

/// One homogeneous detray material slab as a dprop_slab_desc.
template <typename slab_t>
dprop_slab_desc to_slab_desc(const slab_t& slab) {
    const auto& mat = slab.get_material();
    dprop_slab_desc d{};
    d.thickness = static_cast<double>(slab.thickness());
    d.thickness_in_X0 = static_cast<double>(slab.thickness_in_X0());
    d.X0 = static_cast<double>(mat.X0());
    d.molar_electron_density =
        static_cast<double>(mat.molar_electron_density());
    d.mean_excitation_energy =
        static_cast<double>(mat.mean_excitation_energy());
    d.has_density_effect = mat.has_density_effect_data() ? 1u : 0u;
    if (mat.has_density_effect_data()) {
        const auto& de = mat.density_effect_data();
        d.density_a = static_cast<double>(de.get_A_density());
        d.density_m = static_cast<double>(de.get_M_density());
        d.density_x0 = static_cast<double>(de.get_X0_density());
        d.density_x1 = static_cast<double>(de.get_X1_density());
        d.density_c = static_cast<double>(de.get_C_density());
    }
    return d;
}

/// A detray material rod (material/material_rod.hpp) around a line surface
/// as a dprop_slab_desc of kind DPROP_MATERIAL_ROD (thickness = radius).
template <typename rod_t>
dprop_slab_desc to_rod_desc(const rod_t& rod) {
    const auto& mat = rod.get_material();
    dprop_slab_desc d{};
    d.kind = DPROP_MATERIAL_ROD;
    d.thickness = static_cast<double>(rod.radius());
    d.X0 = static_cast<double>(mat.X0());
    d.thickness_in_X0 = d.thickness / d.X0;
    d.molar_electron_density =
        static_cast<double>(mat.molar_electron_density());
    d.mean_excitation_energy =
        static_cast<double>(mat.mean_excitation_energy());
    d.has_density_effect = mat.has_density_effect_data() ? 1u : 0u;
    if (mat.has_density_effect_data()) {
        const auto& de = mat.density_effect_data();
        d.density_a = static_cast<double>(de.get_A_density());
        d.density_m = static_cast<double>(de.get_M_density());
        d.density_x0 = static_cast<double>(de.get_X0_density());
        d.density_x1 = static_cast<double>(de.get_X1_density());
        d.density_c = static_cast<double>(de.get_C_density());
    }
    return d;
}

/// Material-store visitor: homogeneous slabs, rods and 2D material maps.
struct slab_copier {
    template <typename mat_group_t, typename index_t>
    void operator()(const mat_group_t& group, const index_t& idx,
                    flat_detector& out, dprop_surface_desc& sf) const {
        using mat_t = typename mat_group_t::value_type;
        if constexpr (requires(const mat_t& s) {
                          s.thickness_in_X0();
                          s.get_material();
                      }) {
            const dprop_slab_desc d = to_slab_desc(group[idx]);
            sf.material = static_cast<uint32_t>(out.slabs.size());
            out.slabs.push_back(d);
        } else if constexpr (requires(const mat_t& s) {
                                 s.radius();
                                 s.get_material();
                             }) {
            const dprop_slab_desc d = to_rod_desc(group[idx]);
            sf.material = static_cast<uint32_t>(out.slabs.size());
            out.slabs.push_back(d);
        } else if constexpr (detray::concepts::material_map<mat_t>) {
            // 2D material map (material/material_map.hpp): one slab per bin
            if constexpr (mat_t::dim != 2) {
                throw std::runtime_error(
                    "dprop::flatten: volume material maps are not supported "
                    "on the device path");
            }
            const auto g = group[idx];
            using frame_t = typename mat_t::local_frame_type;
            using algebra_t = typename frame_t::algebra_type;
            dprop_grid_desc gd{};
            if constexpr (std::is_same_v<frame_t,
                                         detray::concentric_cylindrical2D<
                                             algebra_t>> ||
                          std::is_same_v<frame_t,
                                         detray::cylindrical2D<algebra_t>>) {
                gd.kind = DPROP_GRID_MATERIAL_CYLINDER;
            } else if constexpr (std::is_same_v<frame_t,
                                                detray::polar2D<algebra_t>>) {
                gd.kind = DPROP_GRID_MATERIAL_DISC;
            } else if constexpr (std::is_same_v<frame_t,
                                                detray::cartesian2D<algebra_t>>) {
                gd.kind = DPROP_GRID_MATERIAL_CARTESIAN;
            } else {
                throw std::runtime_error(
                    "dprop::flatten: unsupported material map frame");
            }
            const auto ax0 = g.template get_axis<0>();
            const auto ax1 = g.template get_axis<1>();
            gd.n_bins[0] = static_cast<uint32_t>(ax0.nbins());
            gd.n_bins[1] = static_cast<uint32_t>(ax1.nbins());
            gd.axis_min[0] = static_cast<double>(ax0.span()[0]);
            gd.axis_max[0] = static_cast<double>(ax0.span()[1]);
            gd.axis_min[1] = static_cast<double>(ax1.span()[0]);
            gd.axis_max[1] = static_cast<double>(ax1.span()[1]);
            gd.transform = sf.transform;
            gd.bin_offset = static_cast<uint32_t>(out.grid_bins.size());
            const std::size_t nb =
                static_cast<std::size_t>(gd.n_bins[0]) * gd.n_bins[1];
            for (std::size_t b = 0; b < nb; ++b) {
                // a bin without an entry holds the empty (zero thickness)
                // slab, which the interactor skips
                dprop_slab_desc d{};
                for (const auto& slab : g.bin(static_cast<detray::dindex>(b))) {
                    d = to_slab_desc(slab);
                }
                out.grid_bins.push_back(static_cast<uint32_t>(out.slabs.size()));
                out.slabs.push_back(d);
            }
            sf.material = static_cast<uint32_t>(out.grids.size());
            sf.material_kind = 1u;
            out.grids.push_back(gd);
        } else {
            throw std::runtime_error(
                "dprop::flatten: only homogeneous material slabs, rods and 2D "
                "material maps are supported on the device path");
        }
    }
};

/// Material-store visitor for a volume's material: a homogeneous material
/// (material/material.hpp, added by homogeneous_volume_material_builder) as
/// a slab of zero thickness; volume material maps are not supported.
struct volume_material_copier {
    template <typename mat_group_t, typename index_t>
    void operator()(const mat_group_t& group, const index_t& idx,
                    flat_detector& out, dprop_volume_desc& vd) const {
        using mat_t = typename mat_group_t::value_type;
        if constexpr (requires(const mat_t& m) {
                          m.X0();
                          m.molar_electron_density();
                          m.mean_excitation_energy();
                      }) {
            const mat_t& mat = group[idx];
            dprop_slab_desc d{};
            d.kind = DPROP_MATERIAL_SLAB;
            d.X0 = static_cast<double>(mat.X0());
            d.molar_electron_density =
                static_cast<double>(mat.molar_electron_density());
            d.mean_excitation_energy =
                static_cast<double>(mat.mean_excitation_energy());
            d.has_density_effect = mat.has_density_effect_data() ? 1u : 0u;
            if (mat.has_density_effect_data()) {
                const auto& de = mat.density_effect_data();
                d.density_a = static_cast<double>(de.get_A_density());
                d.density_m = static_cast<double>(de.get_M_density());
                d.density_x0 = static_cast<double>(de.get_X0_density());
                d.density_x1 = static_cast<double>(de.get_X1_density());
                d.density_c = static_cast<double>(de.get_C_density());
            }
            vd.material = static_cast<uint32_t>(out.slabs.size());
            out.slabs.push_back(d);
        } else {
            throw std::runtime_error(
                "dprop::flatten: only homogeneous volume material is "
                "supported on the device path");
        }
    }
};

/// Accelerator-store visitor: brute-force lists and 2D surface grids.
template <typename detector_t>
struct accel_copier {
    template <typename coll_t, typename index_t>
    void operator()(const coll_t& coll, const index_t& idx,
                    const detector_t& det, flat_detector& out,
                    dprop_volume_desc& vol) const {
        using accel_t = typename coll_t::value_type;
        if constexpr (detray::concepts::surface_accelerator<accel_t> &&
                      requires(const accel_t& a) { a.mask(); }) {
            // 2D spatial surface grid
            const auto g = coll[idx];
            using frame_t = typename accel_t::local_frame_type;
            using algebra_t = typename detector_t::algebra_type;
            dprop_grid_desc gd{};
            if constexpr (std::is_same_v<
                              frame_t,
                              detray::concentric_cylindrical2D<algebra_t>>) {
                gd.kind = DPROP_GRID_CYLINDER;
                gd.radius = static_cast<double>(
                    g.mask()[detray::concentric_cylinder2D::e_r]);
            } else if constexpr (std::is_same_v<frame_t,
                                                detray::polar2D<algebra_t>>) {
                gd.kind = DPROP_GRID_DISC;
            } else {
                throw std::runtime_error(
                    "dprop::flatten: unsupported surface grid frame");
            }
            const auto ax0 = g.template get_axis<0>();
            const auto ax1 = g.template get_axis<1>();
            gd.n_bins[0] = static_cast<uint32_t>(ax0.nbins());
            gd.n_bins[1] = static_cast<uint32_t>(ax1.nbins());
            gd.axis_min[0] = static_cast<double>(ax0.span()[0]);
            gd.axis_max[0] = static_cast<double>(ax0.span()[1]);
            gd.axis_min[1] = static_cast<double>(ax1.span()[0]);
            gd.axis_max[1] = static_cast<double>(ax1.span()[1]);
            gd.transform = vol.transform;
            gd.bin_offset = static_cast<uint32_t>(out.grid_bins.size());
            const std::size_t nb =
                static_cast<std::size_t>(gd.n_bins[0]) * gd.n_bins[1];
            // bin contents in the grid's own order
            std::vector<std::vector<uint32_t>> content(nb);
            std::size_t max_count = 0u;
            for (std::size_t b = 0; b < nb; ++b) {
                for (const auto& sf : g.bin(static_cast<detray::dindex>(b))) {
                    content[b].push_back(static_cast<uint32_t>(sf.index()));
                }
                max_count = std::max(max_count, content[b].size());
            }
            if (max_count <= 1u) {
                gd.multi = 0u;
                for (std::size_t b = 0; b < nb; ++b) {
                    out.grid_bins.push_back(content[b].empty()
                                                ? DPROP_INVALID_INDEX
                                                : content[b][0]);
                }
            } else {
                // ranges first (nb + 1 positions), then the entries
                gd.multi = 1u;
                std::size_t pos = out.grid_bins.size() + nb + 1u;
                for (std::size_t b = 0; b < nb; ++b) {
                    out.grid_bins.push_back(static_cast<uint32_t>(pos));
                    pos += content[b].size();
                }
                out.grid_bins.push_back(static_cast<uint32_t>(pos));
                for (std::size_t b = 0; b < nb; ++b) {
                    out.grid_bins.insert(out.grid_bins.end(),
                                         content[b].begin(), content[b].end());
                }
            }
            vol.grid = static_cast<uint32_t>(out.grids.size());
            out.grids.push_back(gd);
        } else if constexpr (detray::concepts::surface_accelerator<accel_t>) {
            // brute force collection: portals and passives of the volume
            if (vol.bf_end != vol.bf_begin) {
                throw std::runtime_error(
                    "dprop::flatten: more than one brute-force list per "
                    "volume");
            }
            vol.bf_begin = static_cast<uint32_t>(out.bf_surfaces.size());
            for (const auto& sf : coll[idx].all()) {
                out.bf_surfaces.push_back(static_cast<uint32_t>(sf.index()));
            }
            vol.bf_end = static_cast<uint32_t>(out.bf_surfaces.size());
        }
        // volume accelerators (daughter-volume grids) are not searched by the
        // navigator's candidate search (navigation_functions.hpp:73-81)
    }
};

template <typename transform_t, typename algebra_t>
dprop_transform_desc copy_transform(const transform_t& trf) {
    dprop_transform_desc t{};
    const auto& m = trf.matrix();
    const auto& mi = trf.matrix_inverse();
    for (unsigned int c = 0; c < 3u; ++c) {
        for (unsigned int r = 0; r < 3u; ++r) {
            t.rot[c * 3u + r] =
                static_cast<double>(detray::getter::element(m, r, c));
            t.inv_rot[c * 3u + r] =
                static_cast<double>(detray::getter::element(mi, r, c));
        }
        t.translation[c] = static_cast<double>(detray::getter::element(m, c, 3u));
        t.inv_translation[c] =
            static_cast<double>(detray::getter::element(mi, c, 3u));
    }
    return t;
}

}  // namespace adapter_detail

/// Flatten a host detray detector into the tables of the C ABI.
template <typename detector_t>
flat_detector flatten(const detector_t& det) {
    using algebra_t = typename detector_t::algebra_type;
    flat_detector out;

    // transforms (default geometry context)
    const auto& tstore = det.transform_store();
    for (std::size_t i = 0; i < tstore.size(); ++i) {
        out.transforms.push_back(
            adapter_detail::copy_transform<
                std::decay_t<decltype(tstore.at(0))>, algebra_t>(
                tstore.at(static_cast<detray::dindex>(i))));
    }

    // surfaces, their masks and material
    for (const auto& sf : det.surfaces()) {
        dprop_surface_desc d{};
        d.barcode = sf.identifier().value();
        d.transform = static_cast<uint32_t>(sf.transform());
        d.volume = static_cast<uint32_t>(sf.volume());
        d.kind = static_cast<uint8_t>(sf.id());
        d.material = DPROP_INVALID_INDEX;
        det.mask_store().template visit<adapter_detail::mask_copier>(
            sf.mask(), out, d);
        if (sf.has_material()) {
            det.material_store().template visit<adapter_detail::slab_copier>(
                sf.material(), out, d);
        }
        out.surfaces.push_back(d);
    }

    // volumes and their acceleration structures
    for (const auto& v : det.volumes()) {
        dprop_volume_desc vd{};
        vd.transform = static_cast<uint32_t>(v.transform());
        vd.grid = DPROP_INVALID_INDEX;
        vd.material = DPROP_INVALID_INDEX;
        if (v.has_material()) {
            det.material_store()
                .template visit<adapter_detail::volume_material_copier>(
                    v.material(), out, vd);
        }
        const auto& links = v.accel_link();
        for (std::size_t li = 0u; li < links.size(); ++li) {
            const auto& link = links[li];
            if (link.is_invalid()) {
                continue;
            }
            det.accelerator_store()
                .template visit<adapter_detail::accel_copier<detector_t>>(
                    link, det, out, vd);
        }
        out.volumes.push_back(vd);
    }
    return out;
}

}  // namespace dprop
