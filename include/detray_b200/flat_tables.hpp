/*
 * Owning host copy of the flat detector tables of the C ABI
 * (dprop_detector_desc) and their raw file form.
 *
 * flat_detector holds the eight tables dprop_detector_create() uploads;
 * dprop::flatten() (detray_adapter.hpp) fills one from a detray detector,
 * read_raw_tables() from a file written by write_raw_tables().  Needs only
 * the C ABI header.
 */
#pragma once

#include "detray_b200/dprop.h"

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace dprop {

/// Owning flat tables; desc() hands out a view valid while *this lives.
struct flat_detector {
    std::vector<dprop_volume_desc> volumes;
    std::vector<dprop_surface_desc> surfaces;
    std::vector<dprop_mask_desc> masks;
    std::vector<dprop_transform_desc> transforms;
    std::vector<dprop_slab_desc> slabs;
    std::vector<uint32_t> bf_surfaces;
    std::vector<dprop_grid_desc> grids;
    std::vector<uint32_t> grid_bins;

    dprop_detector_desc desc() const {
        dprop_detector_desc d{};
        d.abi_version = DPROP_ABI_VERSION;
        d.n_volumes = static_cast<uint32_t>(volumes.size());
        d.n_surfaces = static_cast<uint32_t>(surfaces.size());
        d.n_masks = static_cast<uint32_t>(masks.size());
        d.n_transforms = static_cast<uint32_t>(transforms.size());
        d.n_slabs = static_cast<uint32_t>(slabs.size());
        d.n_bf_surfaces = static_cast<uint32_t>(bf_surfaces.size());
        d.n_grids = static_cast<uint32_t>(grids.size());
        d.n_grid_bins = static_cast<uint32_t>(grid_bins.size());
        d.volumes = volumes.data();
        d.surfaces = surfaces.data();
        d.masks = masks.data();
        d.transforms = transforms.data();
        d.slabs = slabs.data();
        d.bf_surfaces = bf_surfaces.data();
        d.grids = grids.data();
        d.grid_bins = grid_bins.data();
        return d;
    }
};

/// First word of a raw table file ("DGEO" in little-endian byte order).
constexpr uint32_t k_raw_tables_magic = 0x4f454744u;

/// Write the flat tables to a raw table file: a 12-word u32 header ("DGEO",
/// DPROP_ABI_VERSION, the eight table lengths, two zero words) followed by
/// the tables in declaration order of dprop_detector_desc.  Returns 0 on
/// success.
inline int write_raw_tables(const flat_detector& t, const char* path) {
    std::FILE* f = std::fopen(path, "wb");
    if (!f) {
        return 1;
    }
    const uint32_t header[12] = {k_raw_tables_magic,
                                 DPROP_ABI_VERSION,
                                 static_cast<uint32_t>(t.volumes.size()),
                                 static_cast<uint32_t>(t.surfaces.size()),
                                 static_cast<uint32_t>(t.masks.size()),
                                 static_cast<uint32_t>(t.transforms.size()),
                                 static_cast<uint32_t>(t.slabs.size()),
                                 static_cast<uint32_t>(t.bf_surfaces.size()),
                                 static_cast<uint32_t>(t.grids.size()),
                                 static_cast<uint32_t>(t.grid_bins.size()),
                                 0u,
                                 0u};
    bool ok = std::fwrite(header, sizeof(uint32_t), 12, f) == 12u;
    auto put = [&](const auto& v) {
        if (!v.empty()) {
            ok = ok && std::fwrite(v.data(), sizeof(v[0]), v.size(), f) ==
                           v.size();
        }
    };
    put(t.volumes);
    put(t.surfaces);
    put(t.masks);
    put(t.transforms);
    put(t.slabs);
    put(t.bf_surfaces);
    put(t.grids);
    put(t.grid_bins);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? 0 : 1;
}

/// Read a raw table file written by write_raw_tables.  Returns 0 on
/// success; 1 if the file cannot be read, 2 if it is not a raw table file
/// of this ABI version or is truncated.
inline int read_raw_tables(const char* path, flat_detector& t) {
    std::FILE* f = std::fopen(path, "rb");
    if (!f) {
        return 1;
    }
    uint32_t header[12];
    if (std::fread(header, sizeof(uint32_t), 12, f) != 12u ||
        header[0] != k_raw_tables_magic || header[1] != DPROP_ABI_VERSION) {
        std::fclose(f);
        return 2;
    }
    bool ok = true;
    auto get = [&](auto& v, uint32_t n) {
        v.resize(n);
        if (n != 0u) {
            ok = ok && std::fread(v.data(), sizeof(v[0]), n, f) == n;
        }
    };
    get(t.volumes, header[2]);
    get(t.surfaces, header[3]);
    get(t.masks, header[4]);
    get(t.transforms, header[5]);
    get(t.slabs, header[6]);
    get(t.bf_surfaces, header[7]);
    get(t.grids, header[8]);
    get(t.grid_bins, header[9]);
    std::fclose(f);
    return ok ? 0 : 2;
}

}  // namespace dprop
