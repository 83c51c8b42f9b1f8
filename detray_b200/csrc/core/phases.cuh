// Per-track bodies of the round-based propagation's phases.  A phase loads
// the field groups of slot_soa its segments read, runs them, and stores the
// groups they write; the kernels (rounds_api.cu) wrap these bodies with the
// work queues and warp-level scheduling, and the tests run the same bodies
// on the host in rounds to check that a track driven through them ends
// bit-identical to propagate_track.
//
//   phase_init   propagation start: track state, navigator initialisation
//   fast phase   the loop's light segments, RK steps (with the high-trust
//                navigation update) and the surface actors (transport,
//                material, setter, recorder) until the track needs the
//                volume-level navigation update, or ends
//   phase_nav    the navigation update's cache re-evaluation / volume switch
//   phase_tail   the whole remaining loop inline
#pragma once

#include "slots.cuh"

namespace dprop {

template <bool W>
constexpr uint32_t fast_groups() {
    return g_step | g_meta | g_loop | (W ? g_cyc : 0u);
}
constexpr uint32_t k_nav_load = g_free | g_meta | g_loop;
constexpr uint32_t k_nav_store = g_meta | g_loop;

// The outputs of a finished track (dprop_results fields, in S).
template <typename S>
struct track_outputs {
    uint8_t status;
    uint32_t n_records, n_steps, n_trials, n_isect, n_transport, n_material;
    S path_length;
    S fin[8];
};

template <typename S>
DPROP_HD track_outputs<S> make_outputs(const track_state<S>& ts,
                                       const loop_state<S>& ls,
                                       uint32_t n_records) {
    track_outputs<S> o;
    o.status = track_status(ts, ls.out_of_budget);
    o.n_records = n_records;
    o.n_steps = ts.step.n_steps;
    o.n_trials = ts.step.n_trials;
    o.n_isect = ts.nav.n_isect;
    o.n_transport = ts.n_transport;
    o.n_material = ts.n_material;
    o.path_length = static_cast<S>(ts.step.path_length);
    o.fin[0] = ts.step.pos.x;
    o.fin[1] = ts.step.pos.y;
    o.fin[2] = ts.step.pos.z;
    o.fin[3] = ts.step.time;
    o.fin[4] = ts.step.dir.x;
    o.fin[5] = ts.step.dir.y;
    o.fin[6] = ts.step.dir.z;
    o.fin[7] = ts.step.qop;
    return o;
}

// ------------------------------------------------------------------ init
template <typename S, bool W>
DPROP_HD void phase_init(const slot_soa<S>& s, uint64_t slot, uint32_t track,
                         vec3<S> pos, S time, vec3<S> dir, S qop,
                         const detector_view<S, W>& det,
                         const prop_cfg<S>& cfg) {
    nav_cache<S> cache;
    track_state<S> ts;
    bind_cache(ts.nav, cache);
    loop_state<S> ls;
    init_track_state(ts, pos, time, dir, qop, cfg);
    machine_init(ts, ls, det, cfg);
    store_slot(s, slot, g_step | g_meta | g_bound | g_loop | g_count |
                            (W ? g_cyc : 0u),
               ts, ls);
    for (int k = 0; k <= k_cache; ++k) {
        store_cand(s, slot, k, ts.nav.cand[k]);
    }
    s.rec_count[slot] = 0u;
    s.track[slot] = track;
    s.pc[slot] = ls.pc;
}

// ------------------------------------------------------------------ fast
// The cached candidates a fast-phase track has in registers: the contiguous
// cache indices [lo, hi].  A segment reads at most the current surface, the
// target and the candidate after it (reached and re-intersected in the same
// update), so before each segment the window is grown to cover
// [next - 1, next + 1]; only the entries it covers are loaded and written
// back.
struct cand_window {
    int lo;
    int hi;
};

template <typename S>
DPROP_HD void ensure_cands(const slot_soa<S>& s, uint64_t slot,
                           nav_state<S>& nav, cand_window& w) {
    int a, b;
    cand_range(nav.next - 1, nav.next + 1, a, b);
    for (int k = a; k < w.lo; ++k) {
        load_cand(s, slot, k, nav.cand[k]);
    }
    for (int k = (w.hi + 1 > a ? w.hi + 1 : a); k <= b; ++k) {
        load_cand(s, slot, k, nav.cand[k]);
    }
    w.lo = a < w.lo ? a : w.lo;
    w.hi = b > w.hi ? b : w.hi;
}

// Load the state of the fast phase.
template <typename S, bool W>
DPROP_HD void fast_load(const slot_soa<S>& s, uint64_t slot,
                        track_state<S>& ts, loop_state<S>& ls,
                        cand_window& w) {
    load_slot(s, slot, fast_groups<W>(), ts, ls);
    ls.pc = s.pc[slot];
    w.lo = k_cache + 1;
    w.hi = -1;
    ensure_cands(s, slot, ts.nav, w);
}

// The surface actors inside the fast phase: the track's step, navigation
// and loop state are live, the bound state and counters come from the slot.
template <typename S, bool W>
DPROP_HD void surf_inline(track_state<S>& ts, const slot_soa<S>& s,
                          uint64_t slot, const detector_view<S, W>& det,
                          const field_view<S>& field, const prop_cfg<S>& cfg,
                          record_sink<S>& rec) {
    loop_state<S> unused;
    load_slot(s, slot, g_bound | g_count, ts, unused);
    rec.count = s.rec_count[slot];
    rec.track = rec.stage ? slot : s.track[slot];
    machine_surf(ts, det, field, cfg, rec, no_tape{});
    store_slot(s, slot, g_bound | g_count, ts, unused);
    s.rec_count[slot] = rec.count;
}

// Light segments, the surface actors and at most one RK step; returns the
// next segment.
template <typename S, bool W>
DPROP_HD uint8_t fast_advance(track_state<S>& ts, loop_state<S>& ls,
                              cand_window& w, const slot_soa<S>& s,
                              uint64_t slot, const detector_view<S, W>& det,
                              const field_view<S>& field,
                              const prop_cfg<S>& cfg, record_sink<S>& rec) {
    ensure_cands(s, slot, ts.nav, w);
    uint8_t pc = machine_light(ts, ls, det, cfg, ls.pc);
    if (pc == pc_surf) {
        surf_inline(ts, s, slot, det, field, cfg, rec);
        ensure_cands(s, slot, ts.nav, w);
        pc = machine_light(ts, ls, det, cfg, pc_act_tail);
    }
    if (pc == pc_step) {
        ensure_cands(s, slot, ts.nav, w);
        pc = machine_step(ts, ls, det, field, cfg);
    }
    ls.pc = pc;
    return pc;
}

template <typename S, bool W>
DPROP_HD void fast_store(const slot_soa<S>& s, uint64_t slot,
                         const track_state<S>& ts, const loop_state<S>& ls,
                         const cand_window& w) {
    store_slot(s, slot, fast_groups<W>(), ts, ls);
    for (int k = w.lo; k <= w.hi; ++k) {
        store_cand(s, slot, k, ts.nav.cand[k]);
    }
    s.pc[slot] = ls.pc;
}

// ------------------------------------------------------------------- nav
template <typename S, bool W>
DPROP_HD void phase_nav(const slot_soa<S>& s, uint64_t slot,
                        const detector_view<S, W>& det,
                        const prop_cfg<S>& cfg) {
    nav_cache<S> cache;
    track_state<S> ts;
    bind_cache(ts.nav, cache);
    loop_state<S> ls;
    load_slot(s, slot, k_nav_load, ts, ls);
    for (int k = 0; k <= k_cache; ++k) {
        load_cand(s, slot, k, ts.nav.cand[k]);
    }
    const uint8_t pc = machine_nav(ts, ls, det, cfg);
    store_slot(s, slot, k_nav_store, ts, ls);
    for (int k = 0; k <= k_cache; ++k) {
        store_cand(s, slot, k, ts.nav.cand[k]);
    }
    s.pc[slot] = pc;
}

// ------------------------------------------------------------------ tail
// Load everything, run the loop to its end; returns the outputs (the
// caller writes them at the track's input index).
template <typename S, bool W>
DPROP_HD track_outputs<S> phase_tail(const slot_soa<S>& s, uint64_t slot,
                                     const detector_view<S, W>& det,
                                     const field_view<S>& field,
                                     const prop_cfg<S>& cfg,
                                     record_sink<S>& rec) {
    nav_cache<S> cache;
    track_state<S> ts;
    bind_cache(ts.nav, cache);
    loop_state<S> ls;
    load_slot(s, slot, g_step | g_meta | g_bound | g_loop | g_count |
                           (W ? g_cyc : 0u),
              ts, ls);
    for (int k = 0; k <= k_cache; ++k) {
        load_cand(s, slot, k, ts.nav.cand[k]);
    }
    ls.pc = s.pc[slot];
    rec.count = s.rec_count[slot];
    rec.track = rec.stage ? slot : s.track[slot];
    machine_run(ts, ls, det, field, cfg, rec);
    s.pc[slot] = pc_done;
    s.rec_count[slot] = rec.count;
    return make_outputs(ts, ls, rec.count);
}

// Outputs of a track the fast phase ended: its counters from the slot.
template <typename S>
DPROP_HD track_outputs<S> fast_outputs(const slot_soa<S>& s, uint64_t slot,
                                       track_state<S>& ts,
                                       const loop_state<S>& ls) {
    ts.n_transport = s.n_transport[slot];
    ts.n_material = s.n_material[slot];
    return make_outputs(ts, ls, s.rec_count[slot]);
}

}  // namespace dprop
