// Direct navigation: the track follows a given sequence of surfaces instead
// of searching the volumes (the Kalman-filter step either side of the
// propagation path: fit and smooth along the surfaces of a track candidate).
//
// Reference: direct_navigator, core/include/detray/navigation/
// direct_navigator.hpp:34-304, with the shared helpers update_candidate and
// update_status (navigation/detail/navigation_functions.hpp:99-177).  The
// sequence is the one the surface_sequencer actor collects
// (propagator/actors/surface_sequencer.hpp:24-106): every sensitive or
// material surface the caching navigator reached, i.e. the transported
// records of a propagation.
//
// The state reuses nav_state: cand[0] holds the surface that was reached
// last (current), cand[1] the next surface of the sequence (target); next and
// last stay 1, so the cache is never exhausted and the actors see the same
// state as with the caching navigator.
#pragma once

#include "propagate.cuh"

namespace dprop {

// Surface index of a barcode (geometry::identifier, k_index_mask bits
// 27..47, geometry/identifier.hpp:153-157)
DPROP_HD uint32_t barcode_index(uint64_t bc) {
    return static_cast<uint32_t>((bc >> 27) & 0x1fffffu);
}

template <typename S>
struct direct_navigation {
    const uint64_t* sequence;  // barcodes, slot-major: entry k at k * n + t
    uint64_t n_tracks;
    uint64_t track;
    int32_t length;            // entries of this track's sequence
    int32_t next_external;     // index of the target in the sequence

    DPROP_HD bool forward(const nav_state<S>& nav) const {
        return nav.direction > S(0);
    }
    DPROP_HD bool has_next_external(const nav_state<S>& nav) const {
        return forward(nav) ? next_external != length : next_external != -1;
    }
    template <bool W>
    DPROP_HD uint32_t external(const detector_view<S, W>& det,
                               int32_t k) const {
        const uint32_t sf = barcode_index(
            sequence[static_cast<uint64_t>(k) * n_tracks + track]);
        // an index outside the detector leaves the target unreachable
        return sf < det.n_surfaces ? sf : k_invalid;
    }

    // state::reset: first (forward) or last (backward) entry as target
    template <bool W>
    DPROP_HD void reset(nav_state<S>& nav, const detector_view<S, W>& det) {
        nav.clear_cache();
        next_external = forward(nav) ? 0 : length - 1;
        if (has_next_external(nav)) {
            nav.cand[1].sf = external(det, next_external);
        }
        nav.next = 1;
        nav.last = 1;
    }

    // state::advance: the target becomes the current surface and the next
    // entry of the sequence the target
    template <bool W>
    DPROP_HD void advance(nav_state<S>& nav, const detector_view<S, W>& det) {
        nav.cand[0] = nav.cand[1];
        next_external += forward(nav) ? 1 : -1;
        if (has_next_external(nav)) {
            nav.cand[1].sf = external(det, next_external);
        }
    }

    // direct_navigator::init
    template <bool W>
    DPROP_HD void init(nav_state<S>& nav, const detector_view<S, W>& det,
                       const track_view<S>& trk, const nav_cfg<S>& cfg) {
        nav.clear_cache();
        nav.next = 1;
        nav.last = 1;
        update(nav, det, trk, cfg);
    }

    // direct_navigator::update; returns whether the stepper restarts its
    // step size (a surface was reached)
    template <bool W>
    DPROP_HD bool update(nav_state<S>& nav, const detector_view<S, W>& det,
                         const track_view<S>& trk, const nav_cfg<S>& cfg) {
        if (!has_next_external(nav)) {
            nav.status = e_nav_exit;
            return false;
        }
        if (nav.trust == e_full_trust) {
            return false;
        }
        // every mask accepts the track: the surface is given, not searched
        const S big = static_cast<S>(3.402823466e38f);
        const isect_cfg<S> icfg{big, big, big, cfg.isect.path_tol, -big,
                                true};
        const S ext_tol = limits<S>::max();
        const vec3<S> ro = trk.pos;
        const vec3<S> rd = nav.direction * trk.dir;
        if (!update_candidate(nav.cand[1], det, ro, rd, icfg, ext_tol,
                              nav.n_isect)) {
            nav.abort(e_reason_no_surface);
            return false;
        }
        // update_status with a cache that is never exhausted
        if (fabs(nav.cand[1].path) < cfg.isect.path_tol) {
            nav.status = nav.cand[1].is_portal() ? e_on_portal : e_on_object;
            advance(nav, det);
        } else {
            nav.status = e_towards_object;
        }
        nav.trust = e_full_trust;
        if (nav.status == e_towards_object) {
            return false;
        }
        if (has_next_external(nav) &&
            !update_candidate(nav.cand[1], det, ro, rd, icfg, ext_tol,
                              nav.n_isect)) {
            nav.abort(e_reason_no_surface);
            return false;
        }
        nav.set_volume(det.surfaces[nav.cand[0].sf].volume);
        nav.trust = e_full_trust;
        return true;
    }
};

// Starting point of a direct propagation given as bound parameters on a
// surface (propagator state from bound_track_parameters:
// base_stepper.hpp:84-107 converts them to the free vector on the
// surface): position, direction, time and q/p.
template <typename S, bool W>
DPROP_HD void bound_start(const detector_view<S, W>& det, uint32_t sf_idx,
                          const S bound[6], vec3<S>& pos, vec3<S>& dir,
                          S& time, S& qop) {
    const dev_surface sf = det.surfaces[sf_idx];
    dir = bound_dir(bound[2], bound[3]);
    pos = bound_to_free_pos(det, sf, bound[0], bound[1], dir);
    time = bound[5];
    qop = bound[4];
}

}  // namespace dprop
