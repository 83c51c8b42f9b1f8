/*
 * ORACLE — test infrastructure only.  Never linked into, loaded by or called
 * from the detray-b200 product; only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py use it, and only as the checker / the timed
 * reference CPU implementation.
 *
 * This file compiles the reference detray propagator itself (its headers,
 * where they lie in the reference checkout, plus the host-only vecmem stand-in
 * in oracle/shim) into a shared library with a small C interface:
 *
 *   - ref_build_toy / ref_build_telescope: the reference's own detector
 *     builders (tests/include/detray/test/common/build_toy_detector.hpp:1237,
 *     build_telescope_detector.hpp:187);
 *   - ref_tables: the flat device tables of that detector, produced by the
 *     product's adapter dprop::flatten (include/detray_b200/detray_adapter.hpp);
 *   - ref_propagate: propagator<rk_stepper, caching_navigator, actor_chain<
 *     pathlimit_aborter, parameter_updater<pointwise_material_interactor>,
 *     surface_recorder>>::propagate over a batch of free tracks with OpenMP,
 *     the chain the reference's device tests use
 *     (tests/include/detray/test/device/propagator_test.hpp:84-93,114-168),
 *     writing the same result layout as dprop_propagate_host;
 *   - ref_helix_scan: the reference's navigation-validation scan - every
 *     surface intersected with the track's helix by its helix intersectors
 *     (detector_scanner::run<helix_scan>, tests/include/detray/test/
 *     validation/detector_scanner.hpp:52-140, restated here without its CSV
 *     output dependencies);
 *   - ref_propagate_direct: the same chain with the direct_navigator
 *     (core/include/detray/navigation/direct_navigator.hpp) along given
 *     surface sequences, forward or backward, from free or bound starts.
 *
 * The scalar type is DETRAY_CUSTOM_SCALARTYPE: the recipe builds a double
 * (the correctness oracle) and a float (the CPU timing baseline) library.
 */
#include "detray/definitions/algebra.hpp"
#include "detray/definitions/pdg_particle.hpp"
#include "detray/material/interaction.hpp"
#include "detray/material/material_slab.hpp"
#include "detray/material/predefined_materials.hpp"
#include "detray/navigation/caching_navigator.hpp"
#include "detray/navigation/detail/intersection_kernel.hpp"
#include "detray/navigation/direct_navigator.hpp"
#include "detray/navigation/intersector.hpp"
#include "detray/tracks/helix.hpp"
#include "detray/propagator/actor_chain.hpp"
#include "detray/propagator/actors/aborters.hpp"
#include "detray/propagator/actors/parameter_updater.hpp"
#include "detray/propagator/actors/pointwise_material_interactor.hpp"
#include "detray/propagator/base_actor.hpp"
#include "detray/propagator/propagator.hpp"
#include "detray/propagator/rk_stepper.hpp"
#include "detray/test/common/build_telescope_detector.hpp"
#include "detray/test/common/build_toy_detector.hpp"
#include "detray/test/common/build_wire_chamber.hpp"
#include "detray/tracks/ray.hpp"

#include <vecmem/memory/host_memory_resource.hpp>

#include "detray_b200/detray_adapter.hpp"
#include "ref_field.hpp"

#include <omp.h>

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <variant>
#include <vector>

using namespace detray;

namespace {

using scalar = DETRAY_CUSTOM_SCALARTYPE;
using algebra_t = detray::array<scalar>;

thread_local std::string g_error;

// ---------------------------------------------------------------- detectors
using toy_det_t = detector<toy_metadata<algebra_t>>;
using tel_det_t = detector<telescope_metadata<algebra_t, rectangle2D>>;
using wire_det_t = detector<wire_chamber_metadata<algebra_t>>;

struct det_handle {
    vecmem::host_memory_resource mr;
    std::variant<std::monostate, std::unique_ptr<toy_det_t>,
                 std::unique_ptr<tel_det_t>, std::unique_ptr<wire_det_t>>
        det;
    dprop::flat_detector flat;
    dprop_detector_desc desc{};
};

// ------------------------------------------------------------ field views
// The stepper only calls field.at(x, y, z) and indexes [0..2]
// (core/include/detray/propagator/rk_stepper.hpp:338-344).
struct field_view {
    const oracle_field::field* f;
    std::array<scalar, 3> at(scalar x, scalar y, scalar z) const {
        double b[3];
        f->at(static_cast<double>(x), static_cast<double>(y),
              static_cast<double>(z), b);
        return {static_cast<scalar>(b[0]), static_cast<scalar>(b[1]),
                static_cast<scalar>(b[2])};
    }
};

// --------------------------------------------------- abort reason capture
struct abort_inspector {
    struct void_view : public detray::detail::dbase_view {};
    using view_type = void_view;
    using const_view_type = const void_view;
    const char* last_abort{nullptr};

    constexpr abort_inspector() = default;
    explicit abort_inspector(const void_view&) {}

    template <typename state_t, typename cfg_t, typename p_t, typename d_t>
    void operator()(const state_t&, const cfg_t&, const p_t&, const d_t&,
                    const char*) {}
    template <typename state_t, typename cfg_t, typename p_t, typename d_t,
              typename gen_t>
    void operator()(const state_t&, const cfg_t&, const p_t&, const d_t&,
                    const char* msg, const gen_t& gen) {
        if (msg != nullptr && std::strncmp(msg, "Aborted", 7) == 0) {
            last_abort = gen();
        }
    }
};

// --------------------------------------------------------- the recorder
// Runs after the parameter updater: whenever the navigator reports the
// track on a surface, store the surface barcode, the path length and - if the
// parameter transporter visited this surface - the bound parameters and
// covariance it produced (after the material interactor).
struct record_buffer {
    uint32_t capacity{0};
    uint32_t n{0};
    bool record_all{false};
    struct rec {
        uint64_t barcode;
        std::array<double, 6> bound;
        std::array<double, 21> cov;
        std::array<double, 36> jac;  // accumulated full Jacobian (row-major)
        double path;
        uint8_t flags;
    };
    std::vector<rec> recs;
};

struct surface_recorder : public base_actor {
    struct state {
        record_buffer* buf{nullptr};
        const actor::parameter_updater_state<algebra_t>* updater{nullptr};
    };

    template <typename propagator_state_t>
    void operator()(state& st, propagator_state_t& prop) const {
        // A particle that stopped in material gets q/p = the invalid maximum
        // from the interactor (pointwise_material_interactor.hpp:271-276);
        // the reference would go on stepping with inf/NaN into undefined
        // behaviour (out-of-range table reads, segfaults).  End the track
        // here, after this actor phase's record, as the device path does.
        const bool stopped =
            std::fabs(static_cast<double>(prop.stepping()().qop())) > 1e30;
        const auto& nav = prop.navigation();
        if (!nav.is_on_surface()) {
            if (stopped) {
                prop.navigation().abort("particle stopped in material");
                prop.heartbeat(false);
            }
            return;
        }
        const auto sf = nav.current_surface();
        const bool transported =
            nav.is_on_sensitive() || nav.encountered_sf_material();
        if (!transported && !st.buf->record_all) {
            return;
        }
        record_buffer::rec r{};
        r.barcode = sf.identifier().value();
        r.path = static_cast<double>(prop.stepping().path_length());
        r.flags = 0u;
        if (sf.is_portal()) {
            r.flags |= 2u;
        }
        if (sf.has_material()) {
            r.flags |= 4u;
        }
        const auto& bp = st.updater->bound_params();
        if (transported && bp.surface_link() == sf.identifier()) {
            r.flags |= 1u;
            for (unsigned int i = 0; i < 6u; ++i) {
                r.bound[i] = static_cast<double>(bp[i]);
            }
            const auto& cov = bp.covariance();
            unsigned int k = 0;
            for (unsigned int i = 0; i < 6u; ++i) {
                for (unsigned int j = i; j < 6u; ++j) {
                    r.cov[k++] =
                        static_cast<double>(getter::element(cov, i, j));
                }
            }
            // the reference's product of the surface-to-surface Jacobians
            // (parameter_transporter, parameter_updater.hpp:373-381)
            if (st.updater->has_full_jacobian()) {
                const auto& fj = st.updater->full_jacobian();
                for (unsigned int i = 0; i < 6u; ++i) {
                    for (unsigned int j = 0; j < 6u; ++j) {
                        r.jac[6u * i + j] =
                            static_cast<double>(getter::element(fj, i, j));
                    }
                }
            }
        }
        if (st.buf->n < st.buf->capacity) {
            st.buf->recs.push_back(r);
        }
        ++st.buf->n;
        if (stopped) {
            prop.navigation().abort("particle stopped in material");
            prop.heartbeat(false);
        }
    }
};

template <typename det_t, bool with_interactor, typename nav_inspector_t>
struct prop_types {
    using navigator_t =
        caching_navigator<det_t, navigation::default_cache_size,
                          nav_inspector_t>;
    using stepper_t =
        rk_stepper<field_view, algebra_t, constrained_step<scalar>>;
    using updater_t = std::conditional_t<
        with_interactor,
        actor::parameter_updater<
            algebra_t, actor::pointwise_material_interactor<algebra_t>>,
        actor::parameter_updater<algebra_t>>;
    using chain_t = actor_chain<actor::pathlimit_aborter<scalar>, updater_t,
                                surface_recorder>;
    using propagator_t = propagator<stepper_t, navigator_t, chain_t>;
};

propagation::config to_ref_config(const dprop_config& c) {
    propagation::config p{};
    p.stepping.min_stepsize = c.min_stepsize;
    p.stepping.rk_error_tol = c.rk_error_tol;
    p.stepping.step_constraint = c.step_constraint;
    p.stepping.path_limit = c.path_limit;
    p.stepping.max_rk_updates = c.max_rk_updates;
    p.stepping.use_mean_loss = c.use_mean_loss != 0;
    p.stepping.use_eloss_gradient = c.use_eloss_gradient != 0;
    p.stepping.use_field_gradient = c.use_field_gradient != 0;
    p.stepping.do_covariance_transport = c.do_covariance_transport != 0;
    p.navigation.intersection.min_mask_tolerance = c.min_mask_tolerance;
    p.navigation.intersection.max_mask_tolerance = c.max_mask_tolerance;
    p.navigation.intersection.mask_tolerance_scalor = c.mask_tolerance_scalor;
    p.navigation.intersection.path_tolerance = c.path_tolerance;
    p.navigation.intersection.overstep_tolerance = c.overstep_tolerance;
    p.navigation.search_window = {c.search_window[0], c.search_window[1]};
    p.navigation.accumulated_error = c.accumulated_error;
    p.navigation.n_scattering_stddev = c.n_scattering_stddev;
    p.navigation.estimate_scattering_noise = c.estimate_scattering_noise != 0;
    return p;
}

struct host_results {
    const dprop_results* r;
    uint64_t n;
    template <typename T>
    static void put(void* base, uint64_t i, T v) {
        if (base != nullptr) {
            static_cast<double*>(base)[i] = static_cast<double>(v);
        }
    }
};

/// Write one track's status, final state and records into the results.
template <typename state_t>
void store_results(const dprop_results* out, uint64_t t, uint64_t n,
                   uint8_t status, const record_buffer& buf,
                   const state_t& state, uint32_t cap, double* rec_jac) {
    if (out->status) {
        out->status[t] = status;
    }
    if (out->n_records) {
        out->n_records[t] = buf.n;
    }
    if (out->n_trials) {
        out->n_trials[t] =
            static_cast<uint32_t>(state.stepping().n_total_trials());
    }
    host_results::put(out->path_length, t, state.stepping().path_length());
    const auto& fin = state.stepping()();
    const auto fpos = fin.pos();
    const auto fdir = fin.dir();
    const double fvals[8] = {fpos[0], fpos[1], fpos[2], fin.time(),
                             fdir[0], fdir[1], fdir[2], fin.qop()};
    for (unsigned int k = 0; k < 8u; ++k) {
        host_results::put(out->final_free[k], t, fvals[k]);
    }
    for (uint32_t k = 0; k < static_cast<uint32_t>(buf.recs.size()); ++k) {
        const auto& r = buf.recs[k];
        const uint64_t o = static_cast<uint64_t>(k) * n + t;
        if (out->rec_barcode) {
            out->rec_barcode[o] = r.barcode;
        }
        if (out->rec_flags) {
            out->rec_flags[o] = r.flags;
        }
        host_results::put(out->rec_path, o, r.path);
        for (unsigned int i = 0; i < 6u; ++i) {
            host_results::put(out->rec_bound[i], o, r.bound[i]);
        }
        for (unsigned int i = 0; i < 21u; ++i) {
            host_results::put(out->rec_cov[i], o, r.cov[i]);
        }
        if (rec_jac != nullptr) {
            for (unsigned int i = 0; i < 36u; ++i) {
                rec_jac[(static_cast<uint64_t>(i) * cap + k) * n + t] =
                    r.jac[i];
            }
        }
    }
}

template <typename det_t, bool with_interactor, typename insp_t>
int propagate_impl(const det_t& det, const oracle_field::field& field,
                   const dprop_config& cfg, const double* const trk[8],
                   uint64_t n, const dprop_results* out, int n_threads,
                   int chunk, double* rec_jac) {
    using types = prop_types<det_t, with_interactor, insp_t>;
    using propagator_t = typename types::propagator_t;
    const propagation::config pcfg = to_ref_config(cfg);
    const propagator_t p{pcfg};
    const field_view fview{&field};
    const scalar path_limit = cfg.use_path_limit_aborter
                                  ? static_cast<scalar>(cfg.path_limit)
                                  : std::numeric_limits<scalar>::max();
    const uint32_t cap = cfg.max_records;
    const int ptc_pdg = cfg.pdg;

    if (n_threads > 0) {
        omp_set_num_threads(n_threads);
    }
    const int chunk_sz = chunk > 0 ? chunk : 1;

#pragma omp parallel for schedule(dynamic, chunk_sz)
    for (int64_t ti = 0; ti < static_cast<int64_t>(n); ++ti) {
        const auto t = static_cast<uint64_t>(ti);
        free_track_parameters<algebra_t> track{};
        track.set_pos({static_cast<scalar>(trk[0][t]),
                       static_cast<scalar>(trk[1][t]),
                       static_cast<scalar>(trk[2][t])});
        track.set_time(static_cast<scalar>(trk[3][t]));
        track.set_dir({static_cast<scalar>(trk[4][t]),
                       static_cast<scalar>(trk[5][t]),
                       static_cast<scalar>(trk[6][t])});
        track.set_qop(static_cast<scalar>(trk[7][t]));

        record_buffer buf;
        buf.capacity = cap;
        buf.record_all = cfg.record_all_surfaces != 0;
        buf.recs.reserve(cap);

        typename actor::pathlimit_aborter<scalar>::state pl{path_limit};
        bound_matrix<algebra_t> full_jac =
            matrix::identity<bound_matrix<algebra_t>>();
        actor::parameter_updater_state<algebra_t> us{
            pcfg, rec_jac != nullptr ? &full_jac : nullptr};
        actor::pointwise_material_interactor<algebra_t>::state is{};
        surface_recorder::state rs{&buf, &us};

        typename propagator_t::state state(track, fview, det);
        state.stepping().template set_constraint<step::constraint::e_accuracy>(
            pcfg.stepping.step_constraint);
        // Particle hypothesis: muon (or the configured PDG id) with the
        // charge sign of the track (definitions/pdg_particle.hpp:61-64)
        pdg_particle<scalar> ptc = muon<scalar>();
        if (ptc_pdg == 211 || ptc_pdg == -211) {
            ptc = pion_plus<scalar>();
        } else if (ptc_pdg == 11 || ptc_pdg == -11) {
            ptc = electron<scalar>();
        }
        state.set_particle(update_particle_hypothesis(ptc, track));

        bool ok = false;
        bool failed = false;
        try {
            if constexpr (with_interactor) {
                auto refs = detray::tie(pl, us, is, rs);
                ok = p.propagate(state, refs);
            } else {
                auto refs = detray::tie(pl, us, rs);
                ok = p.propagate(state, refs);
            }
        } catch (const std::exception&) {
            // the reference ran into invalid state (e.g. it keeps stepping a
            // particle that stopped in material and then indexes a table
            // with garbage): report the track as non-finite
            failed = true;
        }
        const auto& fstate = state.stepping()();
        if (!std::isfinite(static_cast<double>(fstate.qop())) ||
            std::fabs(static_cast<double>(fstate.qop())) > 1e30 ||
            !std::isfinite(static_cast<double>(state.stepping().path_length()))) {
            failed = true;
        }

        uint8_t status = DPROP_TRK_EXITED;
        if (failed) {
            status = DPROP_TRK_NONFINITE;
        } else if (!ok) {
            const auto& nav = state.navigation();
            const scalar apl = state.stepping().abs_path_length();
            if (apl >= path_limit) {
                status = DPROP_TRK_PATH_LIMIT;
            } else if constexpr (!std::is_same_v<
                                     insp_t, navigation::void_inspector>) {
                const char* msg = nav.inspector().last_abort;
                if (msg != nullptr &&
                    std::strstr(msg, "stalled") != nullptr) {
                    status = DPROP_TRK_STALLED;
                } else if (msg != nullptr &&
                           std::strstr(msg, "No reachable") != nullptr) {
                    status = DPROP_TRK_NO_SURFACE;
                } else if (msg != nullptr &&
                           std::strstr(msg, "path length") != nullptr) {
                    status = DPROP_TRK_PATH_LIMIT;
                } else {
                    status = DPROP_TRK_NO_SURFACE;
                }
            } else {
                status = DPROP_TRK_NO_SURFACE;
            }
        }

        store_results(out, t, n, status, buf, state, cap, rec_jac);
    }
    return 0;
}

// ------------------------------------------------ direct navigation
// propagator<rk_stepper, direct_navigator, same actor chain> along the given
// surface sequences (barcodes, slot-major [k * n + t]).
template <typename det_t, bool with_interactor>
int propagate_direct_impl(const det_t& det, const oracle_field::field& field,
                          const dprop_config& cfg, const double* const* trk,
                          uint64_t n, const uint64_t* seq,
                          const uint32_t* seq_len, uint32_t max_len,
                          int direction, const uint64_t* start_bc,
                          const double* const* start_bound,
                          const dprop_results* out, int n_threads) {
    using base = prop_types<det_t, with_interactor, navigation::void_inspector>;
    using navigator_t = direct_navigator<det_t>;
    using propagator_t = propagator<typename base::stepper_t, navigator_t,
                                    typename base::chain_t>;
    using surface_t = typename det_t::surface_type;
    const propagation::config pcfg = to_ref_config(cfg);
    const propagator_t p{pcfg};
    const field_view fview{&field};
    const scalar path_limit = cfg.use_path_limit_aborter
                                  ? static_cast<scalar>(cfg.path_limit)
                                  : std::numeric_limits<scalar>::max();
    const uint32_t cap = cfg.max_records;
    if (n_threads > 0) {
        omp_set_num_threads(n_threads);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t ti = 0; ti < static_cast<int64_t>(n); ++ti) {
        const auto t = static_cast<uint64_t>(ti);
        const uint32_t len = seq_len[t] < max_len ? seq_len[t] : max_len;
        std::vector<surface_t> sequence;
        for (uint32_t k = 0; k < len; ++k) {
            const uint64_t bc = seq[static_cast<uint64_t>(k) * n + t];
            sequence.push_back(det.surface(
                static_cast<dindex>((bc >> 27) & 0x1fffffu)));
        }
        if (sequence.empty()) {
            // the reference asserts a non-empty sequence: an empty one ends
            // at once, as its update() does when no target is left
            if (out->status) out->status[t] = DPROP_TRK_EXITED;
            if (out->n_records) out->n_records[t] = 0u;
            continue;
        }
        auto seq_view = vecmem::get_data(sequence);

        record_buffer buf;
        buf.capacity = cap;
        buf.record_all = cfg.record_all_surfaces != 0;
        buf.recs.reserve(cap);
        typename actor::pathlimit_aborter<scalar>::state pl{path_limit};
        actor::parameter_updater_state<algebra_t> us{pcfg};
        actor::pointwise_material_interactor<algebra_t>::state is{};
        surface_recorder::state rs{&buf, &us};

        auto run = [&](auto& state) {
            state.stepping().template set_constraint<
                step::constraint::e_accuracy>(pcfg.stepping.step_constraint);
            if (direction < 0) {
                state.navigation().set_direction(
                    navigation::direction::e_backward);
            }
            state.navigation().reset();
            pdg_particle<scalar> ptc = muon<scalar>();
            if (cfg.pdg == 211 || cfg.pdg == -211) {
                ptc = pion_plus<scalar>();
            } else if (cfg.pdg == 11 || cfg.pdg == -11) {
                ptc = electron<scalar>();
            }
            const auto start = state.stepping()();
            state.set_particle(update_particle_hypothesis(ptc, start));
            bool ok = false;
            bool failed = false;
            try {
                if constexpr (with_interactor) {
                    auto refs = detray::tie(pl, us, is, rs);
                    ok = p.propagate(state, refs);
                } else {
                    auto refs = detray::tie(pl, us, rs);
                    ok = p.propagate(state, refs);
                }
            } catch (const std::exception&) {
                failed = true;
            }
            const auto& fs = state.stepping()();
            if (!std::isfinite(static_cast<double>(fs.qop())) ||
                std::fabs(static_cast<double>(fs.qop())) > 1e30) {
                failed = true;
            }
            uint8_t status = DPROP_TRK_EXITED;
            if (failed) {
                status = DPROP_TRK_NONFINITE;
            } else if (!ok) {
                status = state.stepping().abs_path_length() >= path_limit
                             ? DPROP_TRK_PATH_LIMIT
                             : DPROP_TRK_NO_SURFACE;
            }
            store_results(out, t, n, status, buf, state, cap, nullptr);
        };
        if (start_bc != nullptr) {
            bound_track_parameters<algebra_t> bp{};
            bp.set_surface_link(geometry::identifier{start_bc[t]});
            for (unsigned int i = 0; i < 6u; ++i) {
                bp[i] = static_cast<scalar>(start_bound[i][t]);
            }
            typename propagator_t::state state(bp, fview, det, seq_view);
            run(state);
        } else {
            free_track_parameters<algebra_t> track{};
            track.set_pos({static_cast<scalar>(trk[0][t]),
                           static_cast<scalar>(trk[1][t]),
                           static_cast<scalar>(trk[2][t])});
            track.set_time(static_cast<scalar>(trk[3][t]));
            track.set_dir({static_cast<scalar>(trk[4][t]),
                           static_cast<scalar>(trk[5][t]),
                           static_cast<scalar>(trk[6][t])});
            track.set_qop(static_cast<scalar>(trk[7][t]));
            typename propagator_t::state state(track, fview, det, seq_view);
            run(state);
        }
    }
    return 0;
}

// ------------------------------------------------------------ helix scan
template <typename det_t>
int helix_scan_impl(const det_t& det, const double* bfield,
                    const double* const* trk, uint64_t n, double mask_tol,
                    uint32_t cap, uint8_t* status, uint32_t* n_hits,
                    uint64_t* barcode, double* path, double* loc0,
                    double* loc1, uint16_t* vlink, int n_threads) {
    using surface_t = typename det_t::surface_type;
    using intersection_t =
        intersection2D<surface_t, algebra_t, intersection::contains_pos>;
    using kernel_t = detail::intersection_initialize<intersector>;
    using nav_link_t = typename surface_t::navigation_link;
    const intersection::config icfg{
        .min_mask_tolerance = static_cast<float>(mask_tol),
        .max_mask_tolerance = static_cast<float>(mask_tol),
        .mask_tolerance_scalor = 0.f,
        .overstep_tolerance = 0.f};
    const typename det_t::geometry_context ctx{};
    const dvector3D<algebra_t> B{static_cast<scalar>(bfield[0]),
                                 static_cast<scalar>(bfield[1]),
                                 static_cast<scalar>(bfield[2])};
    if (n_threads > 0) {
        omp_set_num_threads(n_threads);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t ti = 0; ti < static_cast<int64_t>(n); ++ti) {
        const auto t = static_cast<uint64_t>(ti);
        const detail::helix<algebra_t> h(
            {static_cast<scalar>(trk[0][t]), static_cast<scalar>(trk[1][t]),
             static_cast<scalar>(trk[2][t])},
            static_cast<scalar>(trk[3][t]),
            {static_cast<scalar>(trk[4][t]), static_cast<scalar>(trk[5][t]),
             static_cast<scalar>(trk[6][t])},
            static_cast<scalar>(trk[7][t]), B);
        std::vector<intersection_t> trace;
        std::vector<intersection_t> found;
        for (const auto& sf_desc : det.surfaces()) {
            const auto sf = geometry::surface{det, sf_desc};
            try {
                sf.template visit_mask<kernel_t>(found, h, sf_desc,
                                                 det.transform_store(), ctx,
                                                 icfg, scalar{0});
            } catch (const std::exception&) {
                // the reference's root finder throws on a bracket it cannot
                // close; such a surface gives no intersection here
                found.clear();
            }
            for (auto& sfi : found) {
                if (sfi.is_along()) {
                    sfi.set_surface(sf_desc);
                    trace.push_back(sfi);
                }
            }
            found.clear();
        }
        if (trace.empty()) {
            status[t] = DPROP_SCAN_EMPTY;
            n_hits[t] = 0u;
            continue;
        }
        std::stable_sort(trace.begin(), trace.end(),
                         [](const intersection_t& a, const intersection_t& b) {
                             return a < b;
                         });
        std::size_t kept = trace.size();
        for (std::size_t k = 0; k < trace.size(); ++k) {
            if (trace[k].volume_link() ==
                detray::detail::invalid_value<nav_link_t>()) {
                kept = k + 1u;
                break;
            }
        }
        if (kept > cap) {
            status[t] = DPROP_SCAN_OVERFLOW;
            n_hits[t] = static_cast<uint32_t>(kept);
            continue;
        }
        status[t] = DPROP_SCAN_OK;
        n_hits[t] = static_cast<uint32_t>(kept);
        for (std::size_t k = 0; k < kept; ++k) {
            const auto& is = trace[k];
            const uint64_t o = static_cast<uint64_t>(k) * n + t;
            barcode[o] = is.surface().identifier().value();
            path[o] = static_cast<double>(is.path());
            const auto sf = geometry::surface{det, is.surface()};
            const auto p = h.pos(is.path());
            const auto bl = sf.global_to_bound(ctx, p, h.dir(is.path()));
            loc0[o] = static_cast<double>(bl[0]);
            loc1[o] = static_cast<double>(bl[1]);
            vlink[o] = static_cast<uint16_t>(is.volume_link());
        }
    }
    return 0;
}

template <typename det_t>
int dispatch(const det_t& det, const oracle_field::field& f,
             const dprop_config& cfg, const double* const trk[8], uint64_t n,
             const dprop_results* out, int n_threads, int chunk,
             int with_abort_reasons, double* rec_jac) {
    if (cfg.use_material_interactor) {
        if (with_abort_reasons) {
            return propagate_impl<det_t, true, abort_inspector>(
                det, f, cfg, trk, n, out, n_threads, chunk, rec_jac);
        }
        return propagate_impl<det_t, true, navigation::void_inspector>(
            det, f, cfg, trk, n, out, n_threads, chunk, rec_jac);
    }
    if (with_abort_reasons) {
        return propagate_impl<det_t, false, abort_inspector>(
            det, f, cfg, trk, n, out, n_threads, chunk, rec_jac);
    }
    return propagate_impl<det_t, false, navigation::void_inspector>(
        det, f, cfg, trk, n, out, n_threads, chunk, rec_jac);
}

}  // namespace

namespace {

/// A predefined reference material by name (material/predefined_materials.hpp);
/// false for an unknown name.
template <typename F>
bool with_material(const std::string& name, F&& f) {
#define DPROP_REF_MATERIAL(m)      \
    if (name == #m) {              \
        f(m<scalar>());            \
        return true;               \
    }
    DPROP_REF_MATERIAL(hydrogen_liquid)
    DPROP_REF_MATERIAL(hydrogen_gas)
    DPROP_REF_MATERIAL(helium_gas)
    DPROP_REF_MATERIAL(beryllium)
    DPROP_REF_MATERIAL(aluminium)
    DPROP_REF_MATERIAL(silicon)
    DPROP_REF_MATERIAL(silicon_with_ded)
    DPROP_REF_MATERIAL(argon_gas)
    DPROP_REF_MATERIAL(argon_liquid)
    DPROP_REF_MATERIAL(iron)
    DPROP_REF_MATERIAL(iron_with_ded)
    DPROP_REF_MATERIAL(copper)
    DPROP_REF_MATERIAL(copper_with_ded)
    DPROP_REF_MATERIAL(tungsten)
    DPROP_REF_MATERIAL(gold)
    DPROP_REF_MATERIAL(cesium_iodide)
    DPROP_REF_MATERIAL(cesium_iodide_with_ded)
#undef DPROP_REF_MATERIAL
    return false;
}

pdg_particle<scalar> particle_of(int pdg) {
    if (pdg == 11) {
        return electron<scalar>();
    }
    if (pdg == -11) {
        return positron<scalar>();
    }
    if (pdg == 211) {
        return pion_plus<scalar>();
    }
    if (pdg == -13) {
        return antimuon<scalar>();
    }
    return muon<scalar>();
}

}  // namespace

// ======================================================================
extern "C" {

/// Toy geometry parameters (build_toy_detector.hpp:48-213).
typedef struct ref_toy_cfg {
    uint32_t n_brl_layers;
    uint32_t n_edc_layers;
    double module_mat_thickness;   /* mm; <= 0 keeps the default */
    double beampipe_mat_thickness; /* mm; <= 0 keeps the default */
    uint32_t use_material_maps;
    uint32_t pad;
} ref_toy_cfg;

/// Telescope parameters (build_telescope_detector.hpp:36-140).
typedef struct ref_tel_cfg {
    double half_x, half_y;     /* rectangle module half lengths (mm)  */
    const double* positions;   /* module positions along the pilot (mm) */
    uint32_t n_positions;
    uint32_t volume_material;  /* homogeneous volume material: 0 none,
                                  1 cesium iodide (with density-effect
                                  data), 2 iron, 3 liquid argon, 4 silicon
                                  (with density-effect data)               */
    double pilot_dir[3];       /* pilot track direction               */
    double mat_thickness;      /* silicon slab thickness (mm)          */
    double envelope;           /* portal envelope (mm); <= 0 default   */
} ref_tel_cfg;

const char* ref_last_error(void) { return g_error.c_str(); }

int ref_scalar_bytes(void) { return static_cast<int>(sizeof(scalar)); }

int ref_build_toy(const ref_toy_cfg* c, void** out) {
    try {
        auto h = std::make_unique<det_handle>();
        toy_det_config<scalar> cfg{};
        cfg.n_brl_layers(c->n_brl_layers)
            .n_edc_layers(c->n_edc_layers)
            .use_material_maps(c->use_material_maps != 0);
        if (c->module_mat_thickness > 0.) {
            cfg.module_mat_thickness(
                static_cast<scalar>(c->module_mat_thickness));
        }
        if (c->beampipe_mat_thickness > 0.) {
            cfg.beampipe_mat_thickness(
                static_cast<scalar>(c->beampipe_mat_thickness));
        }
        auto [det, names] = build_toy_detector<algebra_t>(h->mr, cfg);
        auto d = std::make_unique<toy_det_t>(std::move(det));
        h->flat = dprop::flatten(*d);
        h->desc = h->flat.desc();
        h->det = std::move(d);
        *out = h.release();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

int ref_build_telescope(const ref_tel_cfg* c, void** out) {
    try {
        auto h = std::make_unique<det_handle>();
        std::vector<scalar> pos;
        for (uint32_t i = 0; i < c->n_positions; ++i) {
            pos.push_back(static_cast<scalar>(c->positions[i]));
        }
        detail::ray<algebra_t> pilot{
            {0.f, 0.f, 0.f},
            0.f,
            {static_cast<scalar>(c->pilot_dir[0]),
             static_cast<scalar>(c->pilot_dir[1]),
             static_cast<scalar>(c->pilot_dir[2])},
            -1.f};
        tel_det_config<algebra_t, rectangle2D> cfg{
            static_cast<scalar>(c->half_x), static_cast<scalar>(c->half_y)};
        cfg.positions(pos).pilot_track(pilot);
        if (c->mat_thickness > 0.) {
            cfg.mat_thickness(static_cast<scalar>(c->mat_thickness));
        }
        if (c->envelope > 0.) {
            cfg.envelope(static_cast<scalar>(c->envelope));
        }
        switch (c->volume_material) {
            case 0u:
                break;
            case 1u:
                cfg.volume_material(cesium_iodide_with_ded<scalar>());
                break;
            case 2u:
                cfg.volume_material(iron<scalar>());
                break;
            case 3u:
                cfg.volume_material(argon_liquid<scalar>());
                break;
            case 4u:
                cfg.volume_material(silicon_with_ded<scalar>());
                break;
            default:
                throw std::runtime_error("unknown volume material code");
        }
        auto [det, names] =
            build_telescope_detector<algebra_t, rectangle2D>(h->mr, cfg);
        auto d = std::make_unique<tel_det_t>(std::move(det));
        h->flat = dprop::flatten(*d);
        h->desc = h->flat.desc();
        h->det = std::move(d);
        *out = h.release();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

/// Wire chamber parameters (build_wire_chamber.hpp:35-145,
/// wire_layer_generator.hpp:33-66).
typedef struct ref_wire_cfg {
    uint32_t n_layers;
    uint32_t square_cells;     /* 1: line_square drift cells, 0: straw tubes */
    double first_layer_inner_radius;
    double half_z;
    double cell_size;
    double stereo_angle;
    double mat_radius;         /* tungsten wire radius (mm)                  */
} ref_wire_cfg;

int ref_build_wire_chamber(const ref_wire_cfg* c, void** out) {
    try {
        auto h = std::make_unique<det_handle>();
        auto build = [&](auto shape_tag) {
            using shape_t = decltype(shape_tag);
            wire_chamber_config<scalar, shape_t> cfg{};
            cfg.n_layers(c->n_layers)
                .first_layer_inner_radius(
                    static_cast<scalar>(c->first_layer_inner_radius))
                .half_z(static_cast<scalar>(c->half_z))
                .cell_size(static_cast<scalar>(c->cell_size))
                .stereo_angle(static_cast<scalar>(c->stereo_angle))
                .mat_radius(static_cast<scalar>(c->mat_radius))
                .do_check(false);
            auto [det, names] = build_wire_chamber<algebra_t>(h->mr, cfg);
            return std::make_unique<wire_det_t>(std::move(det));
        };
        auto d = c->square_cells ? build(line_square{}) : build(line_circular{});
        h->flat = dprop::flatten(*d);
        h->desc = h->flat.desc();
        h->det = std::move(d);
        *out = h.release();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

int ref_tables(void* handle, dprop_detector_desc* out) {
    auto* h = static_cast<det_handle*>(handle);
    *out = h->desc;
    return 0;
}

void ref_destroy(void* handle) { delete static_cast<det_handle*>(handle); }

/// Field descriptor: kind 0 constant (b), kind 1 solenoid map given on an
/// (r, phi, z) grid (same layout as dprop_field_create_grid).
typedef struct ref_field_desc {
    uint32_t kind;
    uint32_t n[3];
    double b[3];
    double lo[3];
    double hi[3];
    const float* values;
} ref_field_desc;

int ref_propagate_jac(void* handle, const ref_field_desc* fd,
                      const dprop_config* cfg, const double* const* tracks,
                      uint64_t n, const dprop_results* out, int n_threads,
                      int chunk, int with_abort_reasons, double* rec_jac);

int ref_propagate(void* handle, const ref_field_desc* fd,
                  const dprop_config* cfg, const double* const* tracks,
                  uint64_t n, const dprop_results* out, int n_threads,
                  int chunk, int with_abort_reasons) {
    return ref_propagate_jac(handle, fd, cfg, tracks, n, out, n_threads, chunk,
                             with_abort_reasons, nullptr);
}

/// ref_propagate plus, per transported record, the reference's accumulated
/// full Jacobian (rec_jac: [36][max_records][n], row-major 6 x 6 elements).
int ref_propagate_jac(void* handle, const ref_field_desc* fd,
                      const dprop_config* cfg, const double* const* tracks,
                      uint64_t n, const dprop_results* out, int n_threads,
                      int chunk, int with_abort_reasons, double* rec_jac) {
    try {
        auto* h = static_cast<det_handle*>(handle);
        oracle_field::field f;
        if (fd->kind == 0u) {
            f.set_constant(fd->b[0], fd->b[1], fd->b[2]);
        } else {
            f.set_grid(fd->lo, fd->hi, fd->n, fd->values);
        }
        if (auto* toy = std::get_if<std::unique_ptr<toy_det_t>>(&h->det)) {
            return dispatch(**toy, f, *cfg, tracks, n, out, n_threads, chunk,
                            with_abort_reasons, rec_jac);
        }
        if (auto* tel = std::get_if<std::unique_ptr<tel_det_t>>(&h->det)) {
            return dispatch(**tel, f, *cfg, tracks, n, out, n_threads, chunk,
                            with_abort_reasons, rec_jac);
        }
        if (auto* wire = std::get_if<std::unique_ptr<wire_det_t>>(&h->det)) {
            return dispatch(**wire, f, *cfg, tracks, n, out, n_threads, chunk,
                            with_abort_reasons, rec_jac);
        }
        g_error = "ref_propagate_jac: empty detector handle";
        return 1;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

/// The reference's helix scan (navigation-validation truth) of every track
/// (tracks: 8 arrays of n doubles) in the constant field b: per track the
/// along-track intersections inside a mask, sorted by |path| and cut after
/// the first world exit, slot-major [k * n + t] with capacity cap; status
/// and n_hits as dprop_scan_results.
int ref_helix_scan(void* handle, const double* b, const double* const* tracks,
                   uint64_t n, double mask_tol, uint32_t cap, uint8_t* status,
                   uint32_t* n_hits, uint64_t* barcode, double* path,
                   double* loc0, double* loc1, uint16_t* vlink,
                   int n_threads) {
    try {
        auto* h = static_cast<det_handle*>(handle);
        auto go = [&](const auto& det) {
            return helix_scan_impl(det, b, tracks, n, mask_tol, cap, status,
                                   n_hits, barcode, path, loc0, loc1, vlink,
                                   n_threads);
        };
        if (auto* toy = std::get_if<std::unique_ptr<toy_det_t>>(&h->det)) {
            return go(**toy);
        }
        if (auto* tel = std::get_if<std::unique_ptr<tel_det_t>>(&h->det)) {
            return go(**tel);
        }
        if (auto* wire = std::get_if<std::unique_ptr<wire_det_t>>(&h->det)) {
            return go(**wire);
        }
        g_error = "ref_helix_scan: empty detector handle";
        return 1;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

/// The reference's direct-navigator propagation along surface sequences
/// (barcodes [max_len * n], slot-major; lengths [n]); direction +1 / -1;
/// start from the free tracks, or - with start_bc - from bound parameters
/// (start_bound: 6 arrays of n) on the surfaces start_bc.  Constant or map
/// field as ref_propagate.
int ref_propagate_direct(void* handle, const ref_field_desc* fd,
                         const dprop_config* cfg, const double* const* tracks,
                         uint64_t n, const uint64_t* seq,
                         const uint32_t* seq_len, uint32_t max_len,
                         int direction, const uint64_t* start_bc,
                         const double* const* start_bound,
                         const dprop_results* out, int n_threads) {
    try {
        auto* h = static_cast<det_handle*>(handle);
        oracle_field::field f;
        if (fd->kind == 0u) {
            f.set_constant(fd->b[0], fd->b[1], fd->b[2]);
        } else {
            f.set_grid(fd->lo, fd->hi, fd->n, fd->values);
        }
        auto go = [&](const auto& det) {
            using det_t = std::decay_t<decltype(det)>;
            if (cfg->use_material_interactor) {
                return propagate_direct_impl<det_t, true>(
                    det, f, *cfg, tracks, n, seq, seq_len, max_len, direction,
                    start_bc, start_bound, out, n_threads);
            }
            return propagate_direct_impl<det_t, false>(
                det, f, *cfg, tracks, n, seq, seq_len, max_len, direction,
                start_bc, start_bound, out, n_threads);
        };
        if (auto* toy = std::get_if<std::unique_ptr<toy_det_t>>(&h->det)) {
            return go(**toy);
        }
        if (auto* tel = std::get_if<std::unique_ptr<tel_det_t>>(&h->det)) {
            return go(**tel);
        }
        if (auto* wire = std::get_if<std::unique_ptr<wire_det_t>>(&h->det)) {
            return go(**wire);
        }
        g_error = "ref_propagate_direct: empty detector handle";
        return 1;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

/// A slab of `thickness` mm of a predefined material as the product's slab
/// descriptor, plus the material's mass density.
int ref_material_slab(const char* name, double thickness,
                      dprop_slab_desc* out, double* mass_density) {
    const bool ok = with_material(name, [&](const auto& mat) {
        const material_slab<scalar> slab(mat, static_cast<scalar>(thickness));
        *out = dprop::adapter_detail::to_slab_desc(slab);
        *mass_density = static_cast<double>(mat.mass_density());
    });
    if (!ok) {
        g_error = std::string("unknown material ") + name;
        return 1;
    }
    return 0;
}

/// The reference's mean Bethe-Bloch stopping power of a particle with
/// momentum p (GeV, detray units) in a predefined material, and its q/p
/// derivative (interaction::compute_bethe_bloch / derive_bethe_bloch,
/// material/interaction.hpp:44-153).  dedx: detray units (energy / length).
int ref_bethe(const char* name, int pdg, double p, double* dedx,
              double* ddedx_dqop) {
    const pdg_particle<scalar> ptc = particle_of(pdg);
    const bool ok = with_material(name, [&](const auto& mat) {
        const scalar qop = ptc.charge() / static_cast<scalar>(p);
        const interaction<scalar> I;
        const detail::relativistic_quantities<scalar> rq(ptc, qop);
        *dedx = static_cast<double>(I.compute_bethe_bloch(mat, ptc, rq));
        *ddedx_dqop = static_cast<double>(I.derive_bethe_bloch(mat, ptc, rq));
    });
    if (!ok) {
        g_error = std::string("unknown material ") + name;
        return 1;
    }
    return 0;
}

/// Evaluate the oracle field at n points (for field-map tests).
int ref_field_eval(const ref_field_desc* fd, const double* xyz, uint64_t n,
                   double* b_out) {
    oracle_field::field f;
    if (fd->kind == 0u) {
        f.set_constant(fd->b[0], fd->b[1], fd->b[2]);
    } else {
        f.set_grid(fd->lo, fd->hi, fd->n, fd->values);
    }
    for (uint64_t i = 0; i < n; ++i) {
        f.at(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], b_out + 3 * i);
    }
    return 0;
}

}  // extern "C"
