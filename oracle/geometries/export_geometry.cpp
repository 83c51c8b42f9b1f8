// Build-time geometry exporter.
//
// Builds the reference's benchmark detectors with detray's own builders
// (tests/include/detray/test/common/build_toy_detector.hpp:1237,
// build_telescope_detector.hpp:187, build_wire_chamber.hpp:147) and writes
// their flattened device tables
// (dprop::flatten, include/detray_b200/detray_adapter.hpp) to a raw table
// file that make_geometries.py packs into the .npz files the product loads.
// It is a detray *user* of the product adapter, compiled against the detray
// headers of a reference checkout; the device library never runs it.
//
// usage: export_geometry toy <n_brl> <n_edc> <module_thickness_mm> <out>
//        export_geometry telescope <half_x> <half_y> <thickness_mm> <out> <x0> [x1 ...]
//        export_geometry wire <n_layers> <square 1|0> <wire_radius_mm> <out>
#include "detray/definitions/algebra.hpp"
#include "detray/test/common/build_telescope_detector.hpp"
#include "detray/test/common/build_toy_detector.hpp"
#include "detray/test/common/build_wire_chamber.hpp"
#include "detray/tracks/ray.hpp"

#include <vecmem/memory/host_memory_resource.hpp>

#include "detray_b200/detray_adapter.hpp"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

using namespace detray;
using algebra_t = detray::array<double>;
using scalar = double;


int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: see source header\n");
        return 2;
    }
    vecmem::host_memory_resource mr;
    const std::string kind = argv[1];
    if (kind == "toy" && (argc == 6 || argc == 7)) {
        // a 7th argument "maps": material maps on the portals
        const bool maps = argc == 7 && std::string(argv[6]) == "maps";
        toy_det_config<scalar> cfg{};
        cfg.n_brl_layers(static_cast<unsigned int>(std::atoi(argv[2])))
            .n_edc_layers(static_cast<unsigned int>(std::atoi(argv[3])))
            .use_material_maps(maps)
            .module_mat_thickness(std::atof(argv[4]));
        auto [det, names] = build_toy_detector<algebra_t>(mr, cfg);
        return dprop::write_raw_tables(dprop::flatten(det), argv[5]);
    }
    if (kind == "telescope" && argc >= 7) {
        std::vector<scalar> pos;
        for (int i = 6; i < argc; ++i) {
            pos.push_back(std::atof(argv[i]));
        }
        tel_det_config<algebra_t, rectangle2D> cfg{std::atof(argv[2]),
                                                   std::atof(argv[3])};
        detail::ray<algebra_t> pilot{{0., 0., 0.}, 0., {1., 0., 0.}, -1.};
        cfg.positions(pos).pilot_track(pilot).mat_thickness(std::atof(argv[4]));
        auto [det, names] = build_telescope_detector<algebra_t, rectangle2D>(mr, cfg);
        return dprop::write_raw_tables(dprop::flatten(det), argv[5]);
    }
    if (kind == "wire" && argc == 6) {
        // 500 mm first layer radius, 1 m half length, 10 mm cells, 50 mrad
        // stereo angle: the builder's defaults
        auto build = [&](auto shape_tag) {
            wire_chamber_config<scalar, decltype(shape_tag)> cfg{};
            cfg.n_layers(static_cast<unsigned int>(std::atoi(argv[2])))
                .mat_radius(std::atof(argv[4]))
                .do_check(false);
            auto [det, names] = build_wire_chamber<algebra_t>(mr, cfg);
            return dprop::write_raw_tables(dprop::flatten(det), argv[5]);
        };
        return std::atoi(argv[3]) ? build(line_square{}) : build(line_circular{});
    }
    std::fprintf(stderr, "bad arguments\n");
    return 2;
}
