// The propagation loop for one track: actors, navigation update and RK
// stepping in the reference's alternating order A N S N A N S N ...
//
// Reference: propagator::propagate, core/include/detray/propagator/
// propagator.hpp:260-400, with the actor chain of the device tests
// (tests/include/detray/test/device/propagator_test.hpp:84-93):
//   pathlimit_aborter -> parameter_updater<pointwise_material_interactor>
// followed by a surface recorder, and the stepper policy
// stepper_rk_policy (navigation/policies.hpp:98-139).
#pragma once

#include <cstring>

#include "adjoint.cuh"

namespace dprop {

template <typename S>
struct prop_cfg {
    step_cfg<S> step;
    nav_cfg<S> nav;
    actor_cfg<S> act;
    S step_constraint;      // stepping::config::step_constraint (accuracy)
    bool record_all;
    uint32_t max_records;
    uint32_t max_iterations;
};

// Words of one staged record: barcode, 6 bound parameters, 21 covariance
// entries, path and flags, padded to a whole number of 16-byte vectors.
template <typename S>
constexpr int staged_record_words() {
    return sizeof(S) == 4 ? 32 : 64;
}

// Where a track writes its records: slot-major arrays, index k * n + t.
// bound and cov point at the caller's arrays of 6 and 21 component pointers
// (in a kernel: the launch parameters, so no per-thread copy is made).
// With stage set, records go instead to a staging area of contiguous
// records, record k of row `track` at (track * capacity + k) *
// staged_record_words(): a lane then writes whole cache lines, where the
// slot-major arrays indexed by the input track would take one sector per
// field when neighbouring lanes hold unrelated input indices
// (unstage_records converts them afterwards).
template <typename S>
struct record_sink {
    uint64_t* barcode;
    S* const* bound;
    S* const* cov;
    S* path;
    uint8_t* flags;
    uint64_t n_tracks;
    uint64_t track;
    uint32_t capacity;
    uint32_t count;
    uint32_t* stage;

    DPROP_HD void write_staged(uint64_t bc, const S* b, const S* c, S p,
                               uint8_t fl) {
        constexpr int nw = staged_record_words<S>();
        constexpr int ws = static_cast<int>(sizeof(S) / 4);
        uint32_t w[nw];
        memcpy(w, &bc, sizeof(bc));
        memcpy(w + 2, b, 6 * sizeof(S));
        memcpy(w + 2 + 6 * ws, c, 21 * sizeof(S));
        memcpy(w + 2 + 27 * ws, &p, sizeof(S));
        w[2 + 28 * ws] = fl;
        for (int i = 3 + 28 * ws; i < nw; ++i) {
            w[i] = 0u;
        }
        uint4* dst = reinterpret_cast<uint4*>(
            stage + (track * capacity + count) * static_cast<uint64_t>(nw));
        for (int i = 0; i < nw / 4; ++i) {
            uint4 v;
            v.x = w[4 * i];
            v.y = w[4 * i + 1];
            v.z = w[4 * i + 2];
            v.w = w[4 * i + 3];
#ifdef __CUDA_ARCH__
            // read once, by the conversion after the propagation: streaming
            // store, so that the records do not push the detector tables,
            // the field map and the slot state out of L2
            __stcs(dst + i, v);
#else
            dst[i] = v;
#endif
        }
    }

    DPROP_HD void write(uint64_t bc, const S* b, const S* c, S p, uint8_t fl) {
        if (stage != nullptr) {
            if (count < capacity) {
                write_staged(bc, b, c, p, fl);
            }
            ++count;
            return;
        }
        if (count < capacity) {
            const uint64_t o = static_cast<uint64_t>(count) * n_tracks + track;
            barcode[o] = bc;
            if (fl & 1u) {
                for (int i = 0; i < 6; ++i) {
                    if (bound[i]) {
                        bound[i][o] = b[i];
                    }
                }
                for (int i = 0; i < 21; ++i) {
                    if (cov[i]) {
                        cov[i][o] = c[i];
                    }
                }
            }
            if (path) {
                path[o] = p;
            }
            if (flags) {
                flags[o] = fl;
            }
        }
        ++count;
    }
};

// Staged record k of staging row `row` written to the slot-major arrays of
// `out` as record k of track `track` (out.stage unset): the writes
// record_sink::write makes, so the results are those of writing directly.
template <typename S>
DPROP_HD void unstage_record(const uint32_t* stage, uint64_t row, uint32_t k,
                             uint64_t track, record_sink<S> out) {
    constexpr int nw = staged_record_words<S>();
    constexpr int ws = static_cast<int>(sizeof(S) / 4);
    const uint4* src = reinterpret_cast<const uint4*>(
        stage + (row * out.capacity + k) * static_cast<uint64_t>(nw));
    uint32_t w[nw];
    for (int i = 0; i < nw / 4; ++i) {
#ifdef __CUDA_ARCH__
        const uint4 v = __ldcs(src + i);
#else
        const uint4 v = src[i];
#endif
        w[4 * i] = v.x;
        w[4 * i + 1] = v.y;
        w[4 * i + 2] = v.z;
        w[4 * i + 3] = v.w;
    }
    uint64_t bc;
    S b[6], c[21], p;
    memcpy(&bc, w, sizeof(bc));
    memcpy(b, w + 2, 6 * sizeof(S));
    memcpy(c, w + 2 + 6 * ws, 21 * sizeof(S));
    memcpy(&p, w + 2 + 27 * ws, sizeof(S));
    out.track = track;
    out.stage = nullptr;
    out.count = k;
    out.write(bc, b, c, p, static_cast<uint8_t>(w[2 + 28 * ws]));
}

// The `count` staged records of staging row `row` (at most the capacity)
// as records of track `track`.
template <typename S>
DPROP_HD void unstage_records(const uint32_t* stage, uint64_t row,
                              uint32_t count, uint64_t track,
                              record_sink<S> out) {
    const uint32_t m = count < out.capacity ? count : out.capacity;
    for (uint32_t k = 0; k < m; ++k) {
        unstage_record(stage, row, k, track, out);
    }
}

// All per-track state of one propagation flow; Grad: the transport Jacobian
// includes the field gradient (use_field_gradient)
template <typename S, bool Grad = false>
struct track_state {
    step_state<S, Grad> step;
    nav_state<S> nav;
    bound_state<S> bound;
    S q;        // particle charge (sign of q/p)
    bool heartbeat;
    uint32_t n_transport;
    uint32_t n_material;
};

template <typename S, bool Grad>
DPROP_HD void init_track_state(track_state<S, Grad>& ts, vec3<S> pos, S time,
                               vec3<S> dir, S qop, const prop_cfg<S>& cfg) {
    step_state<S, Grad>& st = ts.step;
    st.pos = pos;
    st.dir = dir;
    st.qop = qop;
    st.time = time;
    st.path_length = 0.;
    st.abs_path_length = 0.;
    st.step_size = S(0);
    st.next_step_size = S(0);
    st.dtds = {S(0), S(0), S(0)};
    st.dqopds = S(0);
    st.constraint = min_(limits<S>::max(), fabs(cfg.step_constraint));
    st.jac.reset();
    st.n_trials = 0u;
    st.n_steps = 0u;
    ts.nav.reset(0u);
    for (int i = 0; i < 6; ++i) {
        ts.bound.v[i] = S(0);
    }
    for (int i = 0; i < 21; ++i) {
        ts.bound.cov[i] = S(0);
    }
    ts.bound.sf = k_invalid;
    // particle hypothesis with the charge sign of the track
    ts.q = (qop < S(0)) ? S(-1) : S(1);
    ts.heartbeat = false;
    ts.n_transport = 0u;
    ts.n_material = 0u;
}

// The surface actors: parameter_transporter, its observers (material
// interactor, parameter setter) and the surface recorder.  With an
// adjoint_tape (adjoint mode) the derivative data of each transported record
// goes to the tape, and the transport Jacobian restarts at the first
// transported surface as well.
template <typename S, bool W, typename Tape, bool Grad>
DPROP_HD_COLD void run_surface_actors(track_state<S, Grad>& ts,
                                      const detector_view<S, W>& det,
                                      const field_view<S>& field,
                                      const prop_cfg<S>& cfg,
                                      record_sink<S>& rec, const Tape& tape) {
    step_state<S, Grad>& st = ts.step;
    nav_state<S>& nav = ts.nav;
    const uint32_t cur_sf = nav.current().sf;
    const dev_surface dst = det.surfaces[cur_sf];
    const bool on_sensitive =
        nav.status == e_on_object && dst.kind == e_sensitive;
    const bool has_material = dst.material != k_invalid;
    const bool transported = on_sensitive || has_material;
    if (transported) {
        bound_state<S>& b = ts.bound;
        bool update_vector = true;
        S G[4][5];
        vec3<S> dtds_in;
        if constexpr (Tape::enabled) {
            dtds_in = current_dtds(st, field);
            for (int r = 0; r < 4; ++r) {
                for (int c = 0; c < 5; ++c) {
                    G[r][c] = (r == c) ? S(1) : S(0);
                }
            }
        }
        if (b.sf != k_invalid) {
            if (b.sf == cur_sf) {
                update_vector = false;  // already on the departure surface
            } else {
                const dev_surface dep = det.surfaces[b.sf];
                if constexpr (Tape::enabled) {
                    full_jacobian(det, b, dep, dst, st, dtds_in, G);
                } else {
                    full_jacobian(det, b, dep, dst, st, current_dtds(st, field),
                                  G);
                }
                ++ts.n_transport;
                if (fabs(st.path_length) > 0.) {
                    st.jac.reset();
                }
                transport_covariance(G, b.cov);
            }
        } else {
            for (int i = 0; i < 21; ++i) {
                b.cov[i] = S(0);
            }
            for (int i = 0; i < 6; ++i) {
                b.cov[tri6(i, i)] = S(1);
            }
            if constexpr (Tape::enabled) {
                S K[5][7];
                initial_jacobian(det, dst, st, dtds_in, K);
                tape.write_init(K);
                st.jac.reset();
            }
        }
        if (update_vector) {
            free_to_bound(det, dst, st, b.v);
            b.sf = cur_sf;
        }
        // pointwise_material_interactor
        bool success = false;
        S tape_mq = S(1), tape_mc = S(0);
        const S qop_in = b.v[4];
        if (cfg.act.use_interactor && has_material) {
            if constexpr (Tape::enabled) {
                kick_derivatives(det, dst, b.v, cfg.act.mass, ts.q,
                                 nav.direction, tape_mq, tape_mc);
            }
            success = interact(det, dst, b, cfg.act, ts.q, nav.direction);
            ts.n_material += success ? 1u : 0u;
        }
        if constexpr (Tape::enabled) {
            tape.write_record(rec.count, G, tape_mq, tape_mc, dtds_in, qop_in,
                              !update_vector);
        }
        // parameter_setter
        if (success) {
            const vec3<S> d = bound_dir(b.v[2], b.v[3]);
            st.pos = bound_to_free_pos(det, dst, b.v[0], b.v[1], d);
            st.time = b.v[5];
            st.dir = d;
            st.qop = b.v[4];
            if (cfg.act.estimate_noise) {
                estimate_external_tol(nav, b, st, cfg.act, ts.q);
            }
        }
    }
    // surface recorder
    if (transported || cfg.record_all) {
        uint8_t fl = 0u;
        if (transported && ts.bound.sf == cur_sf) {
            fl |= 1u;
        }
        if (dst.kind == e_portal) {
            fl |= 2u;
        }
        if (has_material) {
            fl |= 4u;
        }
        rec.write(dst.barcode, ts.bound.v, ts.bound.cov,
                  static_cast<S>(st.path_length), fl);
    }
}

// pathlimit_aborter (aborters.hpp:23-76): the first actor of the chain.
template <typename S, bool Grad>
DPROP_HD void path_limit_aborter(track_state<S, Grad>& ts, const prop_cfg<S>& cfg) {
    step_state<S, Grad>& st = ts.step;
    nav_state<S>& nav = ts.nav;
    if (!nav.finished()) {
        const S step_limit =
            cfg.act.path_limit - static_cast<S>(fabs(st.abs_path_length));
        if (step_limit <= S(0)) {
            nav.abort(e_reason_path_limit);
            ts.heartbeat = false;
        }
        st.constraint = min_(st.constraint, fabs(step_limit));
    }
}

// Run the actor chain once (propagator.hpp:308).
template <typename S, bool W, typename Tape, bool Grad>
DPROP_HD void run_actors(track_state<S, Grad>& ts, const detector_view<S, W>& det,
                         const field_view<S>& field, const prop_cfg<S>& cfg,
                         record_sink<S>& rec, const Tape& tape) {
    path_limit_aborter(ts, cfg);
    // parameter_transporter and observers only act on surfaces
    if (ts.nav.is_on_surface()) {
        run_surface_actors(ts, det, field, cfg, rec, tape);
    }
}

// stepper_rk_policy: downgrade the navigation trust after a step
template <typename S, bool Grad>
DPROP_HD void rk_policy(nav_state<S>& nav, const step_state<S, Grad>& st) {
    const S d = nav.dist();
    if (fabs(d) <= S(unit::um)) {
        nav.set_high_trust();
        return;
    }
    const S rel = (st.step_size - d) / d;
    if (rel > S(0.1)) {
        nav.set_no_trust();
    } else if (rel > S(0.05)) {
        nav.set_fair_trust();
    } else {
        nav.set_high_trust();
    }
}

// 32-bit key of the exact bit pattern of the state that decides the next
// step: position, direction, q/p, the step sizes and the distance to the
// navigation target.  Equal states give equal keys; different ones almost
// never do.
DPROP_HD uint32_t scalar_bits(float v) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(v);
#else
    uint32_t u;
    memcpy(&u, &v, sizeof(u));
    return u;
#endif
}
DPROP_HD uint32_t scalar_bits(double v) {
#if defined(__CUDA_ARCH__)
    const uint64_t u = static_cast<uint64_t>(__double_as_longlong(v));
#else
    uint64_t u;
    memcpy(&u, &v, sizeof(u));
#endif
    return static_cast<uint32_t>(u) ^ static_cast<uint32_t>(u >> 32);
}
template <typename S, bool Grad>
DPROP_HD uint32_t state_key(const step_state<S, Grad>& st, S target) {
    uint32_t h = scalar_bits(st.pos.x);
    h = h * 0x9e3779b1u ^ scalar_bits(st.pos.y);
    h = h * 0x9e3779b1u ^ scalar_bits(st.pos.z);
    h = h * 0x85ebca6bu ^ scalar_bits(st.dir.x);
    h = h * 0x85ebca6bu ^ scalar_bits(st.dir.y);
    h = h * 0x85ebca6bu ^ scalar_bits(st.dir.z);
    h = h * 0xc2b2ae35u ^ scalar_bits(st.qop);
    h = h * 0x27d4eb2fu ^ scalar_bits(st.step_size);
    h = h * 0x27d4eb2fu ^ scalar_bits(st.next_step_size);
    return h * 0x165667b1u ^ scalar_bits(target);
}

// Exact cycles of the stepping (not in the reference).  A looper whose
// turning point lies a fraction of a um inside a portal cylinder, or which
// grazes a wire cell, can see its target a um or two ahead, step past the
// apex, see it behind and step back, every step longer than the on-surface
// tolerance.  In single precision the state then repeats bit for bit with a
// period of a few steps; the progress check passes on every forward step and
// the reference keeps stepping the cycle until the path-limit aborter ends
// it (millions of steps for the last metre).  The search finds such a cycle
// with Brent's algorithm over state keys, confirms it by meeting the same
// point three times at the same period, and then advances the absolute path,
// the signed path and the time by the whole cycles that still fit below the
// path limit, less one.  The track then runs its last cycles normally and the
// path-limit aborter ends it as in the reference: same status, position,
// direction and momentum, accumulated paths and time up to rounding.  Only
// n_steps / n_trials stay short of the reference's counts.
template <typename S>
struct cycle_search {
    static constexpr uint32_t k_done = 0xffffffffu;
    uint32_t key = 0u;     // state_key of the saved point
    uint32_t lam = 0u;     // steps since the point was saved or last met
    uint32_t power = 1u;   // Brent's window: the saved point moves after it
    uint32_t period = 0u;  // steps between the last two meetings
    uint32_t hits = 0u;    // meetings in a row at that period, or k_done
    double abs0 = 0.;      // accumulators at the last visit of the point
    double path0 = 0.;
    S time0 = S(0);

    template <bool Grad>
    DPROP_HD void save(const step_state<S, Grad>& st) {
        abs0 = st.abs_path_length;
        path0 = st.path_length;
        time0 = st.time;
        lam = 0u;
    }
};

// Called after every step.  Built with DPROP_NO_CYCLE_SKIP it does nothing
// and every cycle is stepped out as the reference does (the test build that
// checks the two agree).
template <typename S, bool Grad>
DPROP_HD void skip_cycles(cycle_search<S>& c, step_state<S, Grad>& st,
                          S target, S path_limit) {
#if defined(DPROP_NO_CYCLE_SKIP)
    return;
#endif
    // Only the states after steps shorter than 1 mm take part: the states
    // of a cycle that has such a step repeat with it, so it is still found,
    // and a cycle of longer steps reaches the path limit within a few
    // thousand steps anyway.  Ordinary steps pay one comparison.
    if (!(fabs(st.step_size) < S(1)) || c.hits == cycle_search<S>::k_done) {
        return;
    }
    const uint32_t key = state_key(st, target);
    ++c.lam;
    if (key == c.key) {
        c.hits = (c.lam == c.period) ? c.hits + 1u : 1u;
        c.period = c.lam;
        if (c.hits < 3u) {
            c.save(st);
            return;
        }
        const double d_abs = st.abs_path_length - c.abs0;
        const double rest =
            static_cast<double>(path_limit) - st.abs_path_length;
        const double k = floor(rest / d_abs) - 1.0;
        if (d_abs > 0. && k >= 1.0) {
            st.abs_path_length += k * d_abs;
            st.path_length += k * (st.path_length - c.path0);
            st.time += static_cast<S>(k) * (st.time - c.time0);
        }
        c.hits = cycle_search<S>::k_done;
        return;
    }
    if (c.lam == c.power) {
        c.key = key;
        c.power = c.power < 0x40000000u ? 2u * c.power : c.power;
        c.period = 0u;
        c.hits = 0u;
        c.save(st);
    }
}

// The caching navigator as the loop's navigation policy
// (navigator_base::init / update, navigation/navigator_base.hpp:56-154).
struct caching_navigation {
    template <typename S, bool W>
    DPROP_HD void init(nav_state<S>& nav, const detector_view<S, W>& det,
                       const track_view<S>& trk, const nav_cfg<S>& cfg) {
        navigator_init(nav, det, trk, cfg);
    }
    template <typename S, bool W>
    DPROP_HD bool update(nav_state<S>& nav, const detector_view<S, W>& det,
                         const track_view<S>& trk, const nav_cfg<S>& cfg) {
        return navigator_update(nav, det, trk, cfg);
    }
};

// dprop_track_status code of a track whose propagation loop has ended
// (propagator.hpp:389-399 and the abort reasons).
template <typename S, bool Grad>
DPROP_HD uint8_t track_status(const track_state<S, Grad>& ts, bool out_of_budget) {
    const nav_state<S>& nav = ts.nav;
    if (out_of_budget) {
        return 4u;  // DPROP_TRK_MAX_ITER
    }
    const bool paused = !ts.heartbeat && nav.is_alive();
    if (nav.finished() || paused) {
        return 0u;  // DPROP_TRK_EXITED
    }
    switch (nav.reason) {
        case e_reason_path_limit:
            return 1u;
        case e_reason_stalled:
            return 2u;
        case e_reason_nonfinite:
            return 6u;  // DPROP_TRK_NONFINITE
        default:
            return 3u;
    }
}

// Propagate one track to the end with the navigation policy Nav (init and
// update of the propagator's navigator); returns a dprop_track_status code.
template <typename S, bool W, typename Tape, typename Nav, bool Grad>
DPROP_HD uint8_t propagate_track_with(Nav& navigator, track_state<S, Grad>& ts,
                                      const detector_view<S, W>& det,
                                      const field_view<S>& field,
                                      const prop_cfg<S>& cfg,
                                      record_sink<S>& rec, const Tape& tape) {
    step_state<S, Grad>& st = ts.step;
    nav_state<S>& nav = ts.nav;

    navigator.init(nav, det, track_view<S>{st.pos, st.dir}, cfg.nav);
    ts.heartbeat = nav.is_alive();
    bool is_init = true;
    double path_prev = 0.;
    uint32_t stall = 0u;
    cycle_search<S> cyc;
    uint32_t i = 0u;
    bool out_of_budget = false;
    for (; (i % 2u == 0u) || ts.heartbeat; ++i) {
        if (i >= cfg.max_iterations) {
            out_of_budget = true;
            break;
        }
        if (i % 2u == 0u) {
            run_actors(ts, det, field, cfg, rec, tape);
            if (!ts.heartbeat) {
                continue;
            }
            path_prev = st.path_length;
        } else {
            const bool reset = nav.is_on_surface() || is_init;
            ts.heartbeat =
                ts.heartbeat &&
                rk_step<S, Grad, W>(st, nav.dist(), cfg.step, reset, field,
                                    det.volume_material(nav.volume), ts.q);
            rk_policy(nav, st);
            if (i > 0u) {
                is_init = false;
            }
            // A state that is no longer finite (a particle stopped in
            // material gets q/p = max, after which the reference computes with
            // inf/NaN) cannot be propagated further: end the track.
            if (!(fabs(st.path_length) < 1e30) || !(fabs(st.qop) < S(1e30)) ||
                !(fabs(st.pos.x) + fabs(st.pos.y) + fabs(st.pos.z) < S(1e30))) {
                ts.heartbeat = false;
                nav.abort(e_reason_nonfinite);
                continue;
            }
            if (fabs(st.path_length) <=
                fabs(path_prev) + static_cast<double>(cfg.nav.isect.path_tol)) {
                if (stall >= 10u) {
                    ts.heartbeat = false;
                    nav.abort(e_reason_stalled);
                }
                ++stall;
            } else {
                stall = 0u;
            }
            // Built into the kernels for detectors with wire surfaces, whose
            // low-pT loopers meet such cycles (about 1 track in 4 000 in the
            // wire chamber, in the solenoid map).  None occurred in 8 M
            // tracks of the toy detector, where the search costs 3-4 % of
            // the propagation time.
            if constexpr (W) {
                skip_cycles(cyc, st, nav.dist(), cfg.act.path_limit);
            }
        }
        is_init = navigator.update(nav, det, track_view<S>{st.pos, st.dir},
                                   cfg.nav) ||
                  is_init;
        ts.heartbeat = ts.heartbeat && nav.is_alive();
    }
    return track_status(ts, out_of_budget);
}

// Propagate one track with the caching navigator.
template <typename S, bool W, typename Tape = no_tape, bool Grad>
DPROP_HD uint8_t propagate_track(track_state<S, Grad>& ts,
                                 const detector_view<S, W>& det,
                                 const field_view<S>& field,
                                 const prop_cfg<S>& cfg, record_sink<S>& rec,
                                 const Tape& tape = Tape{}) {
    caching_navigation navigator;
    return propagate_track_with(navigator, ts, det, field, cfg, rec, tape);
}

}  // namespace dprop
