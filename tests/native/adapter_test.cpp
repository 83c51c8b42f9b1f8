// Test program for the C++ drop-in (include/detray_b200/propagator.hpp):
// propagates a batch of tracks the way the reference's device test does -
// per track a propagator state over the field and detector views and the
// actor states tied together - through dprop::propagator_adapter, and
// writes what the actor states and propagator states hold, for the Python
// test to compare with the ctypes path.
//
//   adapter_test <tables.raw> <config.bin> <tracks.bin> <n> <limit2> <out.bin>
//
// config.bin: a dprop_config; tracks.bin: 8 x n doubles (x, y, z, t, tx,
// ty, tz, q/p, component-major).  Tracks [n/2, n) get a path-limit aborter
// state with limit2, the others one with the configuration's path limit.
// The first 4 tracks are also propagated one call per track; the program
// fails if those differ from the batch.
#include "detray_b200/propagator.hpp"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

using propagator_t = dprop::propagator_adapter<dprop::toy_metadata>;
using aborter_t = dprop::actor::pathlimit_aborter<float>;
using recorder_t = dprop::actor::surface_recorder;
using interactor_t = dprop::actor::pointwise_material_interactor;

struct track_actors {
    recorder_t::state recorder;
    aborter_t::state aborter;
    dprop::actor::parameter_updater_state updater;
    interactor_t::state interactor;

    track_actors(float limit, const dprop::propagation::config& cfg)
        : aborter(limit), updater(cfg) {}
};

bool read_file(const char* path, void* dst, std::size_t bytes) {
    std::FILE* f = std::fopen(path, "rb");
    if (!f) {
        return false;
    }
    const bool ok = std::fread(dst, 1, bytes, f) == bytes;
    std::fclose(f);
    return ok;
}

template <typename T>
void put(std::FILE* f, const T& v) {
    std::fwrite(&v, sizeof(T), 1, f);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 7) {
        std::fprintf(stderr,
                     "usage: adapter_test tables config tracks n limit2 out\n");
        return 2;
    }
    dprop::flat_detector tables;
    if (dprop::read_raw_tables(argv[1], tables) != 0) {
        std::fprintf(stderr, "cannot read tables %s\n", argv[1]);
        return 2;
    }
    dprop::propagation::config cfg{};
    if (!read_file(argv[2], &cfg, sizeof(cfg))) {
        std::fprintf(stderr, "cannot read config %s\n", argv[2]);
        return 2;
    }
    const std::size_t n = std::stoul(argv[4]);
    const float limit2 = std::stof(argv[5]);
    std::vector<double> trk(8 * n);
    if (!read_file(argv[3], trk.data(), trk.size() * sizeof(double))) {
        std::fprintf(stderr, "cannot read tracks %s\n", argv[3]);
        return 2;
    }

    try {
        dprop::detector<dprop::toy_metadata> det(tables);
        // 2 T along z
        dprop::field bfield =
            dprop::field::constant(0., 0., 2. * 0.000299792458);
        propagator_t p{cfg};

        auto track_at = [&](std::size_t t) {
            dprop::free_track_parameters f;
            for (int i = 0; i < 3; ++i) {
                f.pos[i] = trk[i * n + t];
                f.dir[i] = trk[(4 + i) * n + t];
            }
            f.time = trk[3 * n + t];
            f.qop = trk[7 * n + t];
            return f;
        };
        auto limit_of = [&](std::size_t t) {
            return t < n / 2 ? cfg.path_limit : limit2;
        };

        // the batch: states and actor-state tuples of all tracks
        std::vector<track_actors> actors;
        actors.reserve(n);
        std::vector<propagator_t::state> states;
        states.reserve(n);
        using tuple_t = decltype(dprop::tie(
            actors.front().recorder, actors.front().aborter,
            actors.front().updater, actors.front().interactor));
        std::vector<tuple_t> ties;
        ties.reserve(n);
        for (std::size_t t = 0; t < n; ++t) {
            actors.emplace_back(limit_of(t), cfg);
            states.emplace_back(track_at(t), bfield.view(), det.view());
        }
        for (std::size_t t = 0; t < n; ++t) {
            ties.push_back(dprop::tie(actors[t].recorder, actors[t].aborter,
                                      actors[t].updater, actors[t].interactor));
        }
        const std::size_t n_exited = p.propagate(states, ties);

        // one call per track for the first few: same results
        int mismatches = 0;
        for (std::size_t t = 0; t < n && t < 4; ++t) {
            track_actors a(limit_of(t), cfg);
            propagator_t::state s(track_at(t), bfield.view(), det.view());
            const bool ok = p.propagate(
                s, dprop::tie(a.recorder, a.aborter, a.updater, a.interactor));
            const propagator_t::state& b = states[t];
            bool same = ok == b.finished() && s.status() == b.status() &&
                        s.n_steps() == b.n_steps() &&
                        s.path_length() == b.path_length() &&
                        a.recorder.n_records == actors[t].recorder.n_records &&
                        a.recorder.records.size() ==
                            actors[t].recorder.records.size() &&
                        a.interactor.n_interactions ==
                            actors[t].interactor.n_interactions;
            for (std::size_t k = 0; same && k < a.recorder.records.size(); ++k) {
                same = std::memcmp(&a.recorder.records[k],
                                   &actors[t].recorder.records[k],
                                   sizeof(recorder_t::record)) == 0;
            }
            for (int i = 0; same && i < 3; ++i) {
                same = s.stepping().pos[i] == b.stepping().pos[i];
            }
            if (!same) {
                std::fprintf(stderr, "track %zu: single call differs\n", t);
                ++mismatches;
            }
        }

        std::FILE* f = std::fopen(argv[6], "wb");
        if (!f) {
            std::fprintf(stderr, "cannot write %s\n", argv[6]);
            return 2;
        }
        put(f, static_cast<uint64_t>(n_exited));
        for (std::size_t t = 0; t < n; ++t) {
            const propagator_t::state& s = states[t];
            const track_actors& a = actors[t];
            put(f, static_cast<uint32_t>(s.status()));
            put(f, s.n_steps());
            put(f, s.n_trials());
            put(f, a.recorder.n_records);
            put(f, static_cast<uint32_t>(a.recorder.records.size()));
            put(f, a.updater.n_transports);
            put(f, a.interactor.n_interactions);
            put(f, static_cast<uint32_t>(a.updater.has_bound_params()));
            put(f, s.path_length());
            for (int i = 0; i < 3; ++i) put(f, s.stepping().pos[i]);
            put(f, s.stepping().time);
            for (int i = 0; i < 3; ++i) put(f, s.stepping().dir[i]);
            put(f, s.stepping().qop);
            put(f, a.updater.bound_params().surface);
            for (int i = 0; i < 6; ++i) put(f, a.updater.bound_params().vector[i]);
            for (const recorder_t::record& r : a.recorder.records) {
                put(f, r.barcode);
                for (int i = 0; i < 6; ++i) put(f, r.bound[i]);
                for (int i = 0; i < 21; ++i) put(f, r.cov[i]);
                put(f, r.path);
                put(f, static_cast<uint32_t>(r.flags));
            }
        }
        std::fclose(f);
        return mismatches == 0 ? 0 : 1;
    } catch (const dprop::propagation_error& e) {
        std::fprintf(stderr, "propagation error: %s\n", e.what());
        return 3;
    }
}
