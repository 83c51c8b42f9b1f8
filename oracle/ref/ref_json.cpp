/*
 * ORACLE — test infrastructure only, never part of the product.
 *
 * Drives the reference's own JSON detector IO so that the product's reader
 * (detray_b200/io_json.py) can be checked against it:
 *
 *   ref_json write <kind> <dir>
 *       builds a benchmark detector with the reference's builders and writes
 *       it with detray::io::write_detector
 *       (io/include/detray/io/frontend/detector_writer.hpp:25-57):
 *       <name>_geometry.json, _homogeneous_material.json, _material_maps.json
 *       and _surface_grids.json (as the writer decides) under <dir>.
 *   ref_json read <kind> <out> <file.json>...
 *       reads the files with detray::io::read_detector
 *       (io/include/detray/io/frontend/detector_reader.hpp:62-103) into the
 *       detector type of <kind> and writes dprop::flatten() of the result as
 *       a raw table file to <out>.
 *
 * kind: toy | toy_maps | telescope | wire_cells | wire_straws
 *
 * The reference's JSON IO is built on nlohmann/json (pinned to 3.11.3 in the
 * reference's CMakeLists.txt; the Makefile points at a copy of that version).
 */
#include "detray/definitions/algebra.hpp"
#include "detray/io/frontend/detector_reader.hpp"
#include "detray/io/frontend/detector_writer.hpp"
#include "detray/test/common/build_telescope_detector.hpp"
#include "detray/test/common/build_toy_detector.hpp"
#include "detray/test/common/build_wire_chamber.hpp"
#include "detray/tracks/ray.hpp"

#include <vecmem/memory/host_memory_resource.hpp>

#include "detray_b200/detray_adapter.hpp"

#include <cstdio>
#include <exception>
#include <string>
#include <vector>

using namespace detray;
using algebra_t = detray::array<double>;
using scalar = double;

namespace {

template <typename det_t, typename names_t>
int write_json(const det_t& det, const names_t& names, const std::string& dir) {
    auto cfg = io::detector_writer_config{}
                   .format(io::format::json)
                   .path(dir)
                   .replace_files(true)
                   .write_grids(true)
                   .write_material(true);
    io::write_detector(det, names, cfg);
    return 0;
}

template <typename det_t, std::size_t CAP>
int read_json(const std::vector<std::string>& files, const char* out) {
    vecmem::host_memory_resource mr;
    io::detector_reader_config cfg{};
    for (const auto& f : files) {
        cfg.add_file(f);
    }
    cfg.do_check(false);
    auto [det, names] = io::read_detector<det_t, CAP>(mr, cfg);
    return dprop::write_raw_tables(dprop::flatten(det), out);
}

auto build_telescope(vecmem::memory_resource& mr) {
    std::vector<scalar> pos;
    for (int i = 0; i < 10; ++i) {
        pos.push_back(50. * i);
    }
    tel_det_config<algebra_t, rectangle2D> cfg{500., 500.};
    detail::ray<algebra_t> pilot{{0., 0., 0.}, 0., {1., 0., 0.}, -1.};
    cfg.positions(pos).pilot_track(pilot).mat_thickness(0.3);
    return build_telescope_detector<algebra_t, rectangle2D>(mr, cfg);
}

template <typename shape_t>
auto build_wires(vecmem::memory_resource& mr) {
    wire_chamber_config<scalar, shape_t> cfg{};
    cfg.n_layers(10u).mat_radius(0.015).do_check(false);
    return build_wire_chamber<algebra_t>(mr, cfg);
}

auto build_toy(vecmem::memory_resource& mr, bool maps) {
    toy_det_config<scalar> cfg{};
    cfg.n_brl_layers(4u).n_edc_layers(7u).use_material_maps(maps)
        .module_mat_thickness(0.15);
    return build_toy_detector<algebra_t>(mr, cfg);
}

using toy_t = detector<toy_metadata<algebra_t>>;
using tel_t = detector<telescope_metadata<algebra_t, rectangle2D>>;
using wire_t = detector<wire_chamber_metadata<algebra_t>>;

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: see source header\n");
        return 2;
    }
    const std::string mode = argv[1];
    const std::string kind = argv[2];
    try {
        vecmem::host_memory_resource mr;
        if (mode == "write") {
            const std::string dir = argv[3];
            if (kind == "toy" || kind == "toy_maps") {
                auto [det, names] = build_toy(mr, kind == "toy_maps");
                return write_json(det, names, dir);
            }
            if (kind == "telescope") {
                auto [det, names] = build_telescope(mr);
                return write_json(det, names, dir);
            }
            if (kind == "wire_cells") {
                auto [det, names] = build_wires<line_square>(mr);
                return write_json(det, names, dir);
            }
            if (kind == "wire_straws") {
                auto [det, names] = build_wires<line_circular>(mr);
                return write_json(det, names, dir);
            }
        } else if (mode == "read" && argc >= 5) {
            std::vector<std::string> files(argv + 4, argv + argc);
            if (kind == "toy" || kind == "toy_maps") {
                return read_json<toy_t, 1u>(files, argv[3]);
            }
            if (kind == "telescope") {
                return read_json<tel_t, 0u>(files, argv[3]);
            }
            if (kind == "wire_cells" || kind == "wire_straws") {
                return read_json<wire_t, 0u>(files, argv[3]);
            }
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_json: %s\n", e.what());
        return 1;
    }
    std::fprintf(stderr, "bad arguments\n");
    return 2;
}
