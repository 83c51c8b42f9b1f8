// The propagation loop of propagate.cuh as a resumable state machine.
//
// propagate_track_with runs the reference's loop (propagator::propagate,
// core/include/detray/propagator/propagator.hpp:300-387) for one track from
// start to end.  Here the same loop body is cut into segments at the points
// where its work changes character, so that a track can stop after any
// segment, keep its state in device memory and continue later in another
// kernel:
//
//   pc_act        even iteration: iteration budget, path-limit aborter
//   pc_surf       parameter transport, material interaction, parameter
//                 setter and recorder on the surface the track is on
//   pc_act_tail   end of the actor iteration: heartbeat, navigation update
//   pc_nav        the navigation update's volume (re-)initialisation part:
//                 fair/no-trust re-evaluation of the cache, volume switch,
//                 local navigation, loose re-initialisation
//   pc_after_nav  heartbeat from the navigation state, next iteration
//   pc_step       odd iteration: RK step, trust policy, progress checks, the
//                 high-trust navigation update
//   pc_done       the loop has ended
//
// Every segment performs exactly the operations the loop performs between
// the same two points, in the same order, so a track driven segment by
// segment (in any interleaving with other tracks) ends bit-identical to
// propagate_track.  Only the caching navigator is supported.
#pragma once

#include "propagate.cuh"

namespace dprop {

enum machine_pc : uint8_t {
    pc_act = 0,
    pc_surf = 1,
    pc_act_tail = 2,
    pc_nav = 3,
    pc_after_nav = 4,
    pc_step = 5,
    pc_done = 6,
};

// Loop variables of propagate_track_with kept across segments.
template <typename S>
struct loop_state {
    double path_prev;   // path length before the step
    uint32_t i;         // loop iteration
    uint32_t stall;     // consecutive non-advancing steps
    uint8_t pc;         // next segment
    uint8_t nav_mode;   // pc_nav entry: 0 fair/no-trust update, 1 volume
                        // switch / loose re-initialisation only
    bool is_init;
    bool out_of_budget;
    cycle_search<S> cyc;  // exact-cycle search (detectors with wire surfaces)
};

// Start of the loop: navigator initialisation.
template <typename S, bool W>
DPROP_HD void machine_init(track_state<S>& ts, loop_state<S>& ls,
                           const detector_view<S, W>& det,
                           const prop_cfg<S>& cfg) {
    navigator_init(ts.nav, det, track_view<S>{ts.step.pos, ts.step.dir},
                   cfg.nav);
    ts.heartbeat = ts.nav.is_alive();
    ls.path_prev = 0.;
    ls.i = 0u;
    ls.stall = 0u;
    ls.pc = pc_act;
    ls.nav_mode = 0u;
    ls.is_init = true;
    ls.out_of_budget = false;
    ls.cyc = cycle_search<S>{};
}

// Loop condition after ++i: (i % 2 == 0) || heartbeat.
template <typename S>
DPROP_HD uint8_t machine_next(const track_state<S>& ts, loop_state<S>& ls) {
    ++ls.i;
    if (ls.i % 2u == 0u) {
        return pc_act;
    }
    return ts.heartbeat ? pc_step : pc_done;
}

// navigator_update (navigator_base.hpp:121-140 over caching_navigator::
// update_impl) up to the point where it needs the whole candidate cache:
// full trust returns at once, high trust re-intersects the target (and the
// candidate after it when the target is reached).  Returns pc_after_nav when
// the update is complete, pc_nav when the rest runs in machine_nav.
template <typename S, bool W>
DPROP_HD uint8_t machine_nav_fast(track_state<S>& ts, loop_state<S>& ls,
                                  const detector_view<S, W>& det,
                                  const prop_cfg<S>& cfg) {
    nav_state<S>& nav = ts.nav;
    if (nav.trust == e_full_trust) {
        return pc_after_nav;  // the update returned false
    }
    if (nav.trust == e_high_trust &&
        high_trust_update(nav, det, track_view<S>{ts.step.pos, ts.step.dir},
                          cfg.nav)) {
        if (nav.is_on_portal() || nav.trust != e_full_trust ||
            nav.cache_exhausted()) {
            ls.nav_mode = 1u;
            return pc_nav;
        }
        return pc_after_nav;
    }
    ls.nav_mode = 0u;
    return pc_nav;
}

// The rest of navigator_update; is_init |= its result.
template <typename S, bool W>
DPROP_HD uint8_t machine_nav(track_state<S>& ts, loop_state<S>& ls,
                             const detector_view<S, W>& det,
                             const prop_cfg<S>& cfg) {
    nav_state<S>& nav = ts.nav;
    const track_view<S> trk{ts.step.pos, ts.step.dir};
    bool res = false;
    if (ls.nav_mode == 0u) {
        res = fair_or_no_trust_update(nav, det, trk, cfg.nav);
    }
    if (nav.is_on_portal() || nav.trust != e_full_trust ||
        nav.cache_exhausted()) {
        res = finish_update(nav, det, trk, cfg.nav, res);
    }
    ls.is_init = res || ls.is_init;
    return pc_after_nav;
}

template <typename S>
DPROP_HD uint8_t machine_act(track_state<S>& ts, loop_state<S>& ls,
                             const prop_cfg<S>& cfg) {
    if (ls.i >= cfg.max_iterations) {
        ls.out_of_budget = true;
        return pc_done;
    }
    path_limit_aborter(ts, cfg);
    return ts.nav.is_on_surface() ? pc_surf : pc_act_tail;
}

template <typename S, bool W, typename Tape>
DPROP_HD uint8_t machine_surf(track_state<S>& ts,
                              const detector_view<S, W>& det,
                              const field_view<S>& field,
                              const prop_cfg<S>& cfg, record_sink<S>& rec,
                              const Tape& tape) {
    run_surface_actors(ts, det, field, cfg, rec, tape);
    return pc_act_tail;
}

template <typename S, bool W>
DPROP_HD uint8_t machine_act_tail(track_state<S>& ts, loop_state<S>& ls,
                                  const detector_view<S, W>& det,
                                  const prop_cfg<S>& cfg) {
    if (!ts.heartbeat) {
        return machine_next(ts, ls);
    }
    ls.path_prev = ts.step.path_length;
    return machine_nav_fast(ts, ls, det, cfg);
}

template <typename S>
DPROP_HD uint8_t machine_after_nav(track_state<S>& ts, loop_state<S>& ls) {
    ts.heartbeat = ts.heartbeat && ts.nav.is_alive();
    return machine_next(ts, ls);
}

template <typename S, bool W>
DPROP_HD uint8_t machine_step(track_state<S>& ts, loop_state<S>& ls,
                              const detector_view<S, W>& det,
                              const field_view<S>& field,
                              const prop_cfg<S>& cfg) {
    step_state<S>& st = ts.step;
    nav_state<S>& nav = ts.nav;
    if (ls.i >= cfg.max_iterations) {
        ls.out_of_budget = true;
        return pc_done;
    }
    const bool reset = nav.is_on_surface() || ls.is_init;
    ts.heartbeat = ts.heartbeat &&
                   rk_step<S, false, W>(st, nav.dist(), cfg.step, reset, field,
                                        det.volume_material(nav.volume), ts.q);
    rk_policy(nav, st);
    if (ls.i > 0u) {
        ls.is_init = false;
    }
    if (!(fabs(st.path_length) < 1e30) || !(fabs(st.qop) < S(1e30)) ||
        !(fabs(st.pos.x) + fabs(st.pos.y) + fabs(st.pos.z) < S(1e30))) {
        ts.heartbeat = false;
        nav.abort(e_reason_nonfinite);
        return machine_next(ts, ls);
    }
    if (fabs(st.path_length) <=
        fabs(ls.path_prev) + static_cast<double>(cfg.nav.isect.path_tol)) {
        if (ls.stall >= 10u) {
            ts.heartbeat = false;
            nav.abort(e_reason_stalled);
        }
        ++ls.stall;
    } else {
        ls.stall = 0u;
    }
    if constexpr (W) {
        skip_cycles(ls.cyc, st, nav.dist(), cfg.act.path_limit);
    }
    return machine_nav_fast(ts, ls, det, cfg);
}

// Segments that need neither the whole candidate cache nor the surface
// actors: run them until the track reaches pc_step or leaves this class.
template <typename S, bool W>
DPROP_HD uint8_t machine_light(track_state<S>& ts, loop_state<S>& ls,
                               const detector_view<S, W>& det,
                               const prop_cfg<S>& cfg, uint8_t pc) {
    for (int k = 0; k < 8; ++k) {
        if (pc == pc_act) {
            pc = machine_act(ts, ls, cfg);
        } else if (pc == pc_act_tail) {
            pc = machine_act_tail(ts, ls, det, cfg);
        } else if (pc == pc_after_nav) {
            pc = machine_after_nav(ts, ls);
        } else {
            break;
        }
    }
    return pc;
}

// Segments of the step phase (the surface actors run inside it).
DPROP_HD bool machine_is_fast(uint8_t pc) {
    return pc != pc_nav && pc != pc_done;
}

// Run a track from its current segment to the end, every segment inline
// (the form of the loop for the last tracks of a batch).
template <typename S, bool W, typename Tape = no_tape>
DPROP_HD void machine_run(track_state<S>& ts, loop_state<S>& ls,
                          const detector_view<S, W>& det,
                          const field_view<S>& field, const prop_cfg<S>& cfg,
                          record_sink<S>& rec, const Tape& tape = Tape{}) {
    uint8_t pc = ls.pc;
    while (pc != pc_done) {
        pc = machine_light(ts, ls, det, cfg, pc);
        if (pc == pc_step) {
            pc = machine_step(ts, ls, det, field, cfg);
        } else if (pc == pc_surf) {
            pc = machine_surf(ts, det, field, cfg, rec, tape);
        } else if (pc == pc_nav) {
            pc = machine_nav(ts, ls, det, cfg);
        }
    }
    ls.pc = pc_done;
}

}  // namespace dprop
