/*
 * C++ source-level drop-in for the reference's device propagation call.
 *
 * The reference's device code assembles, for each track, a propagator, its
 * state and the actor states, and calls propagate
 * (tests/integration_tests/device/cuda/propagator_cuda_kernel.cu:42-70):
 *
 *   propagator_device_t p{cfg};
 *   pathlimit_aborter_t::state aborter_state{cfg.stepping.path_limit};
 *   actor::parameter_updater_state<algebra> updater_state{cfg};
 *   actor::pointwise_material_interactor<algebra>::state interactor_state{};
 *   auto actor_states = detray::tie(tracer_state, aborter_state,
 *                                   updater_state, interactor_state);
 *   typename propagator_device_t::state state(track, field_data, det);
 *   p.propagate(state, actor_states);
 *
 * with propagator<stepper, navigator, actor_chain>::state(track, field,
 * det) and propagate(state, actor_states)
 * (core/include/detray/propagator/propagator.hpp:89-95, 260-264).
 * dprop::propagator_adapter<metadata> keeps these names and argument
 * meanings over the C ABI (dprop.h):
 *
 *   dprop::propagator_adapter<metadata> p{cfg};
 *   dprop::actor::pathlimit_aborter<float>::state aborter_state{limit};
 *   dprop::actor::parameter_updater_state updater_state{cfg};
 *   dprop::actor::pointwise_material_interactor::state interactor_state{};
 *   dprop::actor::surface_recorder::state recorder_state{};
 *   auto actor_states = dprop::tie(recorder_state, aborter_state,
 *                                  updater_state, interactor_state);
 *   dprop::propagator_adapter<metadata>::state state(track, field.view(),
 *                                                    det.view());
 *   p.propagate(state, actor_states);
 *
 * One propagate(state, actor_states) call runs one track on the GPU.  The
 * batch form propagate(states, actor_states) takes the states and actor
 * states of all tracks - what the reference's kernel launch covers, one
 * thread per track - and runs them in one dprop_propagate_host call.  The
 * actor chain is fixed (path-limit aborter, parameter transporter with the
 * pointwise material interactor and the parameter setter, surface
 * recorder); an actor state in the tuple receives that actor's results,
 * and a chain without an aborter state propagates with the configuration's
 * path limit.
 *
 * Needs only the C ABI header and the C++ standard library; link with
 * libdetray_b200.so.
 */
#pragma once

#include "detray_b200/dprop.h"
#include "detray_b200/flat_tables.hpp"

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace dprop {

/// A failed C ABI call: the status and the library's message.
struct propagation_error : std::runtime_error {
    dprop_status status;
    propagation_error(dprop_status s, const std::string& what)
        : std::runtime_error(what), status(s) {}
};

inline void check(dprop_status s, const char* call) {
    if (s != DPROP_OK) {
        const char* msg = dprop_last_error();
        throw propagation_error(
            s, std::string(call) + ": " + (msg ? msg : "unknown error"));
    }
}

namespace propagation {
/// The reference's propagation::config (stepping, navigation, actor
/// switches) in the flat form of the C ABI.
using config = dprop_config;

inline config default_config() {
    config c{};
    dprop_config_default(&c);
    return c;
}
}  // namespace propagation

/// Free track parameters, detray's free vector [x, y, z, t, tx, ty, tz,
/// q/p] (tracks/free_track_parameters.hpp).
struct free_track_parameters {
    double pos[3]{0., 0., 0.};
    double time{0.};
    double dir[3]{0., 0., 1.};
    double qop{0.};

    free_track_parameters() = default;

    /// From position, time, momentum and charge, as the reference's
    /// free_track_parameters(pos, time, mom, q): direction = mom / |mom|,
    /// q/p = q / |mom|.
    free_track_parameters(const double (&p)[3], double t,
                          const double (&mom)[3], double q)
        : time(t) {
        const double m =
            std::sqrt(mom[0] * mom[0] + mom[1] * mom[1] + mom[2] * mom[2]);
        for (int i = 0; i < 3; ++i) {
            pos[i] = p[i];
            dir[i] = mom[i] / m;
        }
        qop = q / m;
    }

    double p(double q) const { return q / qop; }
};

/// A detector on the device (dprop_detector), uploaded once from flat
/// tables; the reference's detector<metadata> built from its view.
/// metadata_t names the detector family (toy, telescope, wire chamber, or
/// a detray metadata type): it types the views, so that a state cannot be
/// built over a detector of another family.
template <typename metadata_t>
class detector {
public:
    struct view_type {
        const dprop_detector* handle{nullptr};
    };

    explicit detector(const flat_detector& tables, int device = 0) {
        const dprop_detector_desc d = tables.desc();
        check(dprop_detector_create(&d, device, &h_), "dprop_detector_create");
    }
    detector(const detector&) = delete;
    detector& operator=(const detector&) = delete;
    ~detector() {
        if (h_) {
            dprop_detector_destroy(h_);
        }
    }

    view_type view() const { return view_type{h_}; }
    dprop_detector* handle() const { return h_; }

private:
    dprop_detector* h_{nullptr};
};

template <typename metadata_t>
using detector_view = typename detector<metadata_t>::view_type;

/// A magnetic field on the device (dprop_field): constant, or a field map
/// on an (r, phi, z) grid - where the reference plugs a covfie field.
class field {
public:
    struct view_t {
        const dprop_field* handle{nullptr};
    };

    static field constant(double bx, double by, double bz, int device = 0) {
        field f;
        check(dprop_field_create_const(bx, by, bz, device, &f.h_),
              "dprop_field_create_const");
        return f;
    }
    static field grid(const double (&lo)[3], const double (&hi)[3],
                      const uint32_t (&n)[3], const float* values,
                      int device = 0) {
        field f;
        check(dprop_field_create_grid(lo, hi, n, values, device, &f.h_),
              "dprop_field_create_grid");
        return f;
    }
    field(field&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
    field& operator=(field&& o) noexcept {
        std::swap(h_, o.h_);
        return *this;
    }
    field(const field&) = delete;
    field& operator=(const field&) = delete;
    ~field() {
        if (h_) {
            dprop_field_destroy(h_);
        }
    }

    view_t view() const { return view_t{h_}; }

private:
    field() = default;
    dprop_field* h_{nullptr};
};

using field_view = field::view_t;

namespace actor {

/// The reference's pathlimit_aborter<scalar_t> (actors/aborters.hpp:20-73):
/// its state holds the track's path limit.
template <typename scalar_t>
struct pathlimit_aborter {
    struct state {
        scalar_t _path_limit;

        explicit state(scalar_t pl) : _path_limit(pl) {}
        void set_path_limit(scalar_t pl) { _path_limit = pl; }
        scalar_t path_limit() const { return _path_limit; }
    };
};

/// Bound track parameters on a surface: detray's bound vector [loc0, loc1,
/// phi, theta, q/p, t] and the upper triangle of its covariance, row by row.
struct bound_track_parameters {
    uint64_t surface{0};  // barcode (geometry::identifier value)
    double vector[6]{};
    double covariance[21]{};
};

/// The reference's parameter_updater_state (actors/parameter_updater.hpp:
/// 47-120), shared by the parameter transporter, the material interactor
/// and the parameter setter.  After propagate: the bound parameters at the
/// last surface the transporter reached (bound_params(); has_bound_params()
/// is false if it reached none) and the number of transports.
struct parameter_updater_state {
    bool do_covariance_transport{true};
    uint32_t n_transports{0};
    bool has_bound{false};
    bound_track_parameters bound{};

    parameter_updater_state() = default;
    explicit parameter_updater_state(const propagation::config& cfg)
        : do_covariance_transport(cfg.do_covariance_transport != 0) {}

    bool has_bound_params() const { return has_bound; }
    const bound_track_parameters& bound_params() const { return bound; }
};

/// The reference's pointwise_material_interactor
/// (actors/pointwise_material_interactor.hpp): its state receives the
/// number of material interactions.
struct pointwise_material_interactor {
    struct state {
        uint32_t n_interactions{0};
    };
};

/// Records of the surfaces the transporter reached (sensitive or with
/// material; every surface with record_all_surfaces): the device-side
/// recording the reference's device tests make.
struct surface_recorder {
    struct record {
        uint64_t barcode{0};
        double bound[6]{};
        double cov[21]{};   // upper triangle, row by row
        double path{0.};
        uint8_t flags{0};   // bit0 transported, bit1 portal, bit2 material
    };
    struct state {
        std::vector<record> records;  // the first max_records
        uint32_t n_records{0};        // all records, may exceed the capacity
    };
};

}  // namespace actor

/// detray::tie for actor states: a tuple of references.
template <typename... actor_state_t>
std::tuple<actor_state_t&...> tie(actor_state_t&... s) {
    return std::tuple<actor_state_t&...>(s...);
}

namespace adapter_detail {

// pathlimit_aborter<scalar_t>::state for scalar_t in {float, double}
template <typename T>
constexpr bool aborter_state_v =
    std::is_same_v<T, actor::pathlimit_aborter<float>::state> ||
    std::is_same_v<T, actor::pathlimit_aborter<double>::state>;

// Calls f(s) on every element of a tuple of references (the tuple is
// copied, the states it refers to are not).
template <typename tuple_t, typename F, std::size_t... I>
void for_each_ref(tuple_t& t, F&& f, std::index_sequence<I...>) {
    (f(std::get<I>(t)), ...);
}
template <typename... A, typename F>
void for_each_state(std::tuple<A&...> t, F&& f) {
    for_each_ref(t, f, std::index_sequence_for<A...>{});
}

}  // namespace adapter_detail

/// The propagator over the C ABI, typed by the detector family.
template <typename metadata_t>
class propagator_adapter {
public:
    using detector_type = detector<metadata_t>;
    using detector_view_type = detector_view<metadata_t>;
    using field_view_type = field_view;

    /// The state of one propagation flow (propagator::state_base,
    /// propagator.hpp:64-95): built from the track, the field view and the
    /// detector view.  stepping() holds the free parameters - the start
    /// before propagate, the end after it.
    class state {
    public:
        state(const free_track_parameters& track, const field_view_type& f,
              const detector_view_type& det)
            : m_track(track), m_field(f), m_det(det) {}

        const free_track_parameters& stepping() const { return m_track; }
        /// dprop_track_status of the last propagate (DPROP_TRK_NOT_RUN
        /// before).
        dprop_track_status status() const { return m_status; }
        /// The navigation left the world: what propagate() returned.
        bool finished() const { return m_status == DPROP_TRK_EXITED; }
        double path_length() const { return m_path_length; }
        uint32_t n_steps() const { return m_n_steps; }
        uint32_t n_trials() const { return m_n_trials; }
        uint32_t n_intersections() const { return m_n_isect; }

    private:
        friend class propagator_adapter;
        free_track_parameters m_track;
        field_view_type m_field;
        detector_view_type m_det;
        dprop_track_status m_status{DPROP_TRK_NOT_RUN};
        double m_path_length{0.};
        uint32_t m_n_steps{0}, m_n_trials{0}, m_n_isect{0};
    };

    /// The library's default launch: direction-sorted tracks, the round-based
    /// method.
    static dprop_launch default_launch() {
        dprop_launch lc{};
        lc.method = DPROP_METHOD_PERSISTENT;
        lc.sort_tracks = 1u;
        return lc;
    }

    explicit propagator_adapter(
        const propagation::config& cfg = propagation::default_config(),
        const dprop_launch& launch = default_launch())
        : m_cfg(cfg), m_launch(launch) {}

    const propagation::config& config() const { return m_cfg; }
    const dprop_launch& launch() const { return m_launch; }

    /// propagator::propagate (propagator.hpp:260-399) for one track: true if
    /// the navigation left the world.
    template <typename... actor_state_t>
    bool propagate(state& s, std::tuple<actor_state_t&...> actor_states) const {
        state* one[1] = {&s};
        run(one, 1u, [&](std::size_t) { return actor_states; });
        return s.finished();
    }
    bool propagate(state& s) const { return propagate(s, std::tuple<>{}); }

    /// The reference's kernel launch over a batch: states[i] with
    /// actor_states[i] (tuples of references made by dprop::tie), in one
    /// dprop_propagate_host call per distinct path limit.  Returns the
    /// number of tracks that left the world.
    template <typename actor_states_t>
    std::size_t propagate(std::vector<state>& states,
                          std::vector<actor_states_t>& actor_states) const {
        if (actor_states.size() != states.size()) {
            throw propagation_error(DPROP_E_INVALID,
                                    "propagate: one actor-state tuple per "
                                    "state");
        }
        std::vector<state*> ptr(states.size());
        for (std::size_t i = 0; i < states.size(); ++i) {
            ptr[i] = &states[i];
        }
        run(ptr.data(), ptr.size(),
            [&](std::size_t i) { return actor_states[i]; });
        return count_finished(states);
    }
    std::size_t propagate(std::vector<state>& states) const {
        std::vector<state*> ptr(states.size());
        for (std::size_t i = 0; i < states.size(); ++i) {
            ptr[i] = &states[i];
        }
        run(ptr.data(), ptr.size(),
            [](std::size_t) { return std::tuple<>{}; });
        return count_finished(states);
    }

private:
    static std::size_t count_finished(const std::vector<state>& states) {
        std::size_t k = 0;
        for (const state& s : states) {
            k += s.finished() ? 1u : 0u;
        }
        return k;
    }

    // The path limit a track's actor chain asks for: its aborter state's,
    // or the configuration's (chain without an aborter state: flag 0).
    template <typename tuple_t>
    static std::pair<int, float> limit_of(tuple_t t, const dprop_config& c) {
        std::pair<int, float> r{0, c.path_limit};
        adapter_detail::for_each_state(t, [&](auto& a) {
            using T = std::decay_t<decltype(a)>;
            if constexpr (adapter_detail::aborter_state_v<T>) {
                r = {1, static_cast<float>(a.path_limit())};
            }
        });
        return r;
    }

    template <typename actors_of_t>
    void run(state* const* st, std::size_t n, actors_of_t&& actors_of) const {
        if (n == 0u) {
            return;
        }
        for (std::size_t i = 1; i < n; ++i) {
            if (st[i]->m_det.handle != st[0]->m_det.handle ||
                st[i]->m_field.handle != st[0]->m_field.handle) {
                throw propagation_error(DPROP_E_INVALID,
                                        "propagate: the states of a batch "
                                        "share one detector and one field");
            }
        }
        if (st[0]->m_det.handle == nullptr || st[0]->m_field.handle == nullptr) {
            throw propagation_error(DPROP_E_INVALID,
                                    "propagate: state without detector or "
                                    "field");
        }
        // groups of equal path limit, in first-appearance order
        std::vector<std::pair<std::pair<int, float>, std::vector<std::size_t>>>
            groups;
        for (std::size_t i = 0; i < n; ++i) {
            const std::pair<int, float> key = limit_of(actors_of(i), m_cfg);
            std::size_t g = 0;
            while (g < groups.size() && groups[g].first != key) {
                ++g;
            }
            if (g == groups.size()) {
                groups.push_back({key, {}});
            }
            groups[g].second.push_back(i);
        }
        for (const auto& grp : groups) {
            dprop_config c = m_cfg;
            if (grp.first.first) {
                c.use_path_limit_aborter = 1u;
                c.path_limit = grp.first.second;
            }
            run_group(c, st, grp.second, actors_of);
        }
    }

    template <typename actors_of_t>
    void run_group(const dprop_config& c, state* const* st,
                   const std::vector<std::size_t>& idx,
                   actors_of_t& actors_of) const {
        const std::size_t m = idx.size();
        // records are fetched only when a recorder or updater state asks
        bool want_records = false;
        for (std::size_t j = 0; j < m && !want_records; ++j) {
            adapter_detail::for_each_state(actors_of(idx[j]), [&](auto& a) {
                using T = std::decay_t<decltype(a)>;
                want_records =
                    want_records ||
                    std::is_same_v<T, actor::surface_recorder::state> ||
                    std::is_same_v<T, actor::parameter_updater_state>;
            });
        }
        std::vector<double> trk(8 * m);
        for (std::size_t j = 0; j < m; ++j) {
            const free_track_parameters& t = st[idx[j]]->m_track;
            for (int i = 0; i < 3; ++i) {
                trk[i * m + j] = t.pos[i];
                trk[(4 + i) * m + j] = t.dir[i];
            }
            trk[3 * m + j] = t.time;
            trk[7 * m + j] = t.qop;
        }
        dprop_tracks tr{};
        for (int i = 0; i < 3; ++i) {
            tr.pos[i] = &trk[i * m];
            tr.dir[i] = &trk[(4 + i) * m];
        }
        tr.time = &trk[3 * m];
        tr.qop = &trk[7 * m];

        const std::size_t cap = want_records ? c.max_records : 0u;
        std::vector<uint8_t> status(m, DPROP_TRK_NOT_RUN);
        std::vector<uint32_t> n_rec(m), n_steps(m), n_trials(m), n_isect(m),
            n_trans(m), n_mat(m);
        std::vector<float> path(m), fin(8 * m);
        std::vector<uint64_t> offs(want_records ? m + 1 : 0);
        std::vector<uint64_t> rbc(cap * m);
        std::vector<float> rb(6 * cap * m), rc(21 * cap * m), rp(cap * m);
        std::vector<uint8_t> rf(cap * m);
        dprop_results r{};
        r.status = status.data();
        r.n_records = n_rec.data();
        r.n_steps = n_steps.data();
        r.n_trials = n_trials.data();
        r.path_length = path.data();
        for (int i = 0; i < 8; ++i) {
            r.final_free[i] = &fin[i * m];
        }
        r.n_intersections = n_isect.data();
        r.n_transports = n_trans.data();
        r.n_material = n_mat.data();
        if (want_records) {
            r.rec_barcode = rbc.data();
            for (int i = 0; i < 6; ++i) {
                r.rec_bound[i] = &rb[i * cap * m];
            }
            for (int i = 0; i < 21; ++i) {
                r.rec_cov[i] = &rc[i * cap * m];
            }
            r.rec_path = rp.data();
            r.rec_flags = rf.data();
            r.rec_offsets = offs.data();
        }
        check(dprop_propagate_host(&c, &m_launch, st[idx[0]]->m_det.handle,
                                   st[idx[0]]->m_field.handle, &tr, &r, m),
              "dprop_propagate_host");

        for (std::size_t j = 0; j < m; ++j) {
            state& s = *st[idx[j]];
            s.m_status = static_cast<dprop_track_status>(status[j]);
            s.m_path_length = path[j];
            s.m_n_steps = n_steps[j];
            s.m_n_trials = n_trials[j];
            s.m_n_isect = n_isect[j];
            if (s.m_status != DPROP_TRK_NOT_RUN) {
                for (int i = 0; i < 3; ++i) {
                    s.m_track.pos[i] = fin[i * m + j];
                    s.m_track.dir[i] = fin[(4 + i) * m + j];
                }
                s.m_track.time = fin[3 * m + j];
                s.m_track.qop = fin[7 * m + j];
            }
            const uint64_t b = want_records ? offs[j] : 0u;
            const uint64_t e = want_records ? offs[j + 1] : 0u;
            auto rec_at = [&](uint64_t o) {
                actor::surface_recorder::record x;
                x.barcode = rbc[o];
                for (int i = 0; i < 6; ++i) {
                    x.bound[i] = rb[i * cap * m + o];
                }
                for (int i = 0; i < 21; ++i) {
                    x.cov[i] = rc[i * cap * m + o];
                }
                x.path = rp[o];
                x.flags = rf[o];
                return x;
            };
            adapter_detail::for_each_state(actors_of(idx[j]), [&](auto& a) {
                using T = std::decay_t<decltype(a)>;
                if constexpr (std::is_same_v<T, actor::surface_recorder::state>) {
                    a.n_records = n_rec[j];
                    a.records.clear();
                    for (uint64_t o = b; o < e; ++o) {
                        a.records.push_back(rec_at(o));
                    }
                } else if constexpr (std::is_same_v<
                                         T, actor::parameter_updater_state>) {
                    a.n_transports = n_trans[j];
                    a.has_bound = false;
                    for (uint64_t o = e; o > b; --o) {
                        if (rf[o - 1] & 1u) {
                            const actor::surface_recorder::record x =
                                rec_at(o - 1);
                            a.has_bound = true;
                            a.bound.surface = x.barcode;
                            for (int i = 0; i < 6; ++i) {
                                a.bound.vector[i] = x.bound[i];
                            }
                            for (int i = 0; i < 21; ++i) {
                                a.bound.covariance[i] = x.cov[i];
                            }
                            break;
                        }
                    }
                } else if constexpr (std::is_same_v<
                                         T, actor::pointwise_material_interactor::
                                                state>) {
                    a.n_interactions = n_mat[j];
                }
            });
        }
    }

    propagation::config m_cfg;
    dprop_launch m_launch;
};

/// Detector families of the bundled geometries (metadata tags).
struct toy_metadata {};
struct telescope_metadata {};
struct wire_chamber_metadata {};

}  // namespace dprop
