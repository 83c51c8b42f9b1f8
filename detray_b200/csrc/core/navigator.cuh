// Navigation: the candidate cache, its trust-level update and the volume
// search, one track per thread.
//
// Follows the reference's caching navigator step for step so that the
// sequence of surfaces a track crosses is the same:
//   cache state         navigation/navigation_state.hpp:67-668
//   insert              navigation/caching_navigator.hpp:149-229
//   update_impl         navigation/caching_navigator.hpp:250-369
//   init / update       navigation/navigator_base.hpp:56-154
//   candidate_search    navigation/detail/navigation_functions.hpp:26-81
//   update_candidate    navigation/detail/navigation_functions.hpp:99-129
//   update_status       navigation/detail/navigation_functions.hpp:147-177
//   local_navigation    navigation/detail/navigation_functions.hpp:193-246
//   volume_switch       navigation/detail/navigation_functions.hpp:264-288
//   init_loose_cfg      navigation/detail/navigation_functions.hpp:304-331
//   intersection kernel navigation/detail/intersection_kernel.hpp:24-272
//   grid search         navigation/accelerators/spatial_grid.hpp:100-201,
//                       utils/grid/detail/axis_binning.hpp, axis_bounds.hpp,
//                       utils/grid/detail/bin_view.hpp (axis 0 outer loop)
#pragma once

#include "geometry.cuh"

namespace dprop {

constexpr int k_cache = 8;  // navigation::default_cache_size

enum nav_status : int8_t {
    e_nav_abort = -3,
    e_nav_exit = -2,
    e_nav_unknown = -1,
    e_towards_object = 0,
    e_on_object = 1,
    e_on_portal = 2,
};

enum trust_level : uint8_t {
    e_no_trust = 0,
    e_fair_trust = 1,
    e_high_trust = 3,
    e_full_trust = 4,
};

enum abort_reason : uint8_t {
    e_reason_none = 0,
    e_reason_path_limit = 1,
    e_reason_stalled = 2,
    e_reason_no_surface = 3,
    e_reason_nonfinite = 4,
};

template <typename S>
struct nav_cfg {
    isect_cfg<S> isect;
    uint32_t win0, win1;
};

template <typename S>
struct nav_state {
    // k_cache candidates plus one sentinel slot: when the last cached
    // candidate is reached the next index points one past the cache, and a
    // read there (which the reference does on its fixed-size array) finds
    // an unreachable candidate instead of leaving the state.
    // The cache lives outside this struct, in an array of k_cache + 1
    // candidates the owner binds here (nav_cache): indexed with the
    // run-time cache index, an array inside the state would make the
    // compiler keep the whole per-track state in the thread's stack instead
    // of registers.
    candidate<S>* cand;
    int8_t next;
    int8_t last;
    int8_t status;
    uint8_t trust;
    uint32_t volume;
    S external_tol;
    S direction;  // +1 forward, -1 backward
    uint8_t reason;
    uint32_t n_isect;  // ray-surface intersections evaluated

    DPROP_HD void reset(uint32_t vol) {
        for (int i = 0; i <= k_cache; ++i) {
            cand[i] = invalid_candidate<S>();
        }
        next = 0;
        last = -1;
        status = e_nav_unknown;
        trust = e_no_trust;
        volume = vol;
        external_tol = S(0);
        direction = S(1);
        reason = e_reason_none;
        n_isect = 0u;
    }
    DPROP_HD bool is_alive() const { return status > e_nav_unknown; }
    DPROP_HD bool finished() const { return status == e_nav_exit; }
    DPROP_HD bool is_on_surface() const {
        return status == e_on_object || status == e_on_portal;
    }
    DPROP_HD bool is_on_portal() const { return status == e_on_portal; }
    DPROP_HD int n_candidates() const { return last - next + 1; }
    DPROP_HD bool cache_exhausted() const { return n_candidates() == 0; }
    DPROP_HD int begin_index() const {
        return (is_on_surface() && next >= 1) ? next - 1 : next;
    }
    DPROP_HD int end_index() const { return last + 1; }
    DPROP_HD candidate<S>& current() { return cand[next - 1]; }
    DPROP_HD const candidate<S>& current() const { return cand[next - 1]; }
    DPROP_HD candidate<S>& target() { return cand[next]; }
    DPROP_HD const candidate<S>& target() const { return cand[next]; }
    // distance to the next candidate along the navigation direction
    DPROP_HD S dist() const { return direction * cand[next].path; }
    DPROP_HD void set_no_trust() { trust = e_no_trust; }
    DPROP_HD void set_high_trust() {
        trust = trust < e_high_trust ? trust : e_high_trust;
    }
    DPROP_HD void set_fair_trust() {
        trust = trust < e_fair_trust ? trust : e_fair_trust;
    }
    DPROP_HD void set_volume(uint32_t v) {
        if (v != volume) {
            set_no_trust();
        }
        volume = v;
    }
    DPROP_HD void clear_cache() {
        for (int i = 0; i < k_cache; ++i) {
            cand[i].path = limits<S>::max();
        }
        next = 0;
        last = -1;
    }
    DPROP_HD void abort(uint8_t why) {
        status = e_nav_abort;
        reason = why;
    }
};

// Storage of a candidate cache (k_cache candidates and the sentinel); bind
// it to a state with bind_cache before the state is used.
template <typename S>
struct nav_cache {
    candidate<S> c[k_cache + 1];
};

template <typename S>
DPROP_HD void bind_cache(nav_state<S>& nav, nav_cache<S>& cache) {
    nav.cand = cache.c;
}

// Track position and direction seen by the navigator
template <typename S>
struct track_view {
    vec3<S> pos;
    vec3<S> dir;
};

#if defined(DPROP_TRACE) && !defined(__CUDA_ARCH__)
}  // namespace dprop
#include <cstdio>
namespace dprop {
template <typename S>
void nav_trace(const nav_state<S>& nav, const char* msg, vec3<S> p) {
    std::printf("[%s] st=%d trust=%d vol=%u pos=(%.4f %.4f %.4f)\n", msg,
                (int)nav.status, (int)nav.trust, (unsigned)nav.volume,
                (double)p.x, (double)p.y, (double)p.z);
    for (int i = 0; i < k_cache; ++i) {
        const candidate<S>& c = nav.cand[i];
        std::printf("   c%d sf=%u path=%.6f st=%d vl=%u\n", i,
                    c.sf == k_invalid ? 9999999u : c.sf,
                    c.path > S(1e30) ? -1.0 : (double)c.path, (int)c.status,
                    (unsigned)c.volume_link);
    }
}
#define DPROP_NAV_TRACE(nav, msg, p) nav_trace(nav, msg, p)
#else
#define DPROP_NAV_TRACE(nav, msg, p)
#endif

// --------------------------------------------------------- cache insert
template <typename S>
DPROP_HD void nav_insert(nav_state<S>& nav, const candidate<S>& nc) {
    // upper_bound over [begin, end) with |path| ordering
    const int b = nav.begin_index();
    const int e = nav.end_index();
    int pos = e;
    const S apath = fabs(nc.path);
    for (int i = b; i < e; ++i) {
        if (apath < fabs(nav.cand[i].path)) {
            pos = i;
            break;
        }
    }
    if (pos == k_cache) {
        return;  // too far away to be cached
    }
    if (nav.n_candidates() == 0) {
        nav.cand[0] = nc;
        nav.last = static_cast<int8_t>(nav.last + 1);
        return;
    }
    const S um = S(unit::um);
    // the same surface (same index <=> same barcode) at an overlapping path
    // is not added twice
    if ((nav.cand[pos].sf == nc.sf &&
         fabs(nav.cand[pos].path - nc.path) <= um) ||
        (pos > 0 && nav.cand[pos - 1].sf == nc.sf &&
         fabs(nav.cand[pos - 1].path - nc.path) <= um)) {
        return;
    }
    const int shift_max = k_cache - 2;
    const int shift_begin = nav.last < shift_max ? nav.last : shift_max;
    // prefer sensitives over portals and direct over edge hits
    if (fabs(nav.cand[pos].path - nc.path) <= um &&
        (nc.is_edge() || nc.is_portal())) {
        ++pos;
        pos = pos > shift_begin ? shift_begin : pos;
    }
    for (int i = shift_begin; i >= pos; --i) {
        nav.cand[i + 1] = nav.cand[i];
    }
    nav.cand[pos] = nc;
    const int nl = nav.last + 1;
    nav.last = static_cast<int8_t>(nl < k_cache - 1 ? nl : k_cache - 1);
}

// -------------------------------------------- intersection_initialize
// Intersect one surface with the tangential ray and insert the result(s).
template <typename S, bool W>
DPROP_HD_LEAF void candidate_search(nav_state<S>& nav, const detector_view<S, W>& det,
                               uint32_t sf_idx, vec3<S> ro, vec3<S> rd,
                               const isect_cfg<S>& cfg) {
    const dev_surface sf = det.surfaces[sf_idx];
    const dev_transform<S>& trf = det.transforms[sf.transform];
    const uint32_t m0 = sf.mask_begin;
    const uint32_t m1 = sf.mask_begin + sf.n_masks;
    ++nav.n_isect;
    if (sf.shape == e_cylinder) {
        isect_point<S> ips[2];
        intersect_cylinder(ro, rd, trf, det.masks[m0].v[0], ips);
        if (!ip_valid(ips[0].path) && !ip_valid(ips[1].path)) {
            return;
        }
        for (uint32_t mi = m0; mi < m1; ++mi) {
            candidate<S> is = invalid_candidate<S>();
            int n_found = 0;
            for (int i = 0; i < 2; ++i) {
                resolve_mask<W>(is, ips[i], sf_idx, sf, det.masks[mi], trf, cfg,
                             nav.external_tol);
                if (is.is_probably_inside()) {
                    nav_insert(nav, is);
                    ++n_found;
                }
                if (n_found == 2) {
                    return;
                }
            }
        }
        return;
    }
    isect_point<S> ip;
    if (sf.shape == e_concentric_cylinder) {
        ip = intersect_portal_cylinder(ro, rd, det.masks[m0].v[0],
                                       cfg.overstep_tol);
    } else if (W && sf.shape == e_line) {
        ip = intersect_line(ro, rd, trf);
    } else {
        ip = intersect_plane(ro, rd, trf);
    }
    if (!ip_valid(ip.path)) {
        return;
    }
    for (uint32_t mi = m0; mi < m1; ++mi) {
        candidate<S> is = invalid_candidate<S>();
        resolve_mask<W>(is, ip, sf_idx, sf, det.masks[mi], trf, cfg,
                     nav.external_tol);
        if (is.is_probably_inside()) {
            nav_insert(nav, is);
            return;
        }
    }
}

// ------------------------------------------------- intersection_update
template <typename S, bool W>
DPROP_HD_LEAF bool update_candidate(candidate<S>& c, const detector_view<S, W>& det,
                               vec3<S> ro, vec3<S> rd, const isect_cfg<S>& cfg,
                               S external_tol, uint32_t& n_isect) {
    if (c.sf == k_invalid) {
        return false;
    }
    ++n_isect;
    const uint32_t sf_idx = c.sf;
    const dev_surface sf = det.surfaces[sf_idx];
    const dev_transform<S>& trf = det.transforms[sf.transform];
    const uint32_t m0 = sf.mask_begin;
    const uint32_t m1 = sf.mask_begin + sf.n_masks;
    isect_point<S> ip;
    if (sf.shape == e_cylinder) {
        isect_point<S> ips[2];
        intersect_cylinder(ro, rd, trf, det.masks[m0].v[0], ips);
        if (!ip_valid(ips[0].path) && !ip_valid(ips[1].path)) {
            return false;
        }
        ip = ips[0];
    } else {
        if (sf.shape == e_concentric_cylinder) {
            ip = intersect_portal_cylinder(ro, rd, det.masks[m0].v[0],
                                           cfg.overstep_tol);
        } else if (W && sf.shape == e_line) {
            ip = intersect_line(ro, rd, trf);
        } else {
            ip = intersect_plane(ro, rd, trf);
        }
        if (!ip_valid(ip.path)) {
            return false;
        }
    }
    for (uint32_t mi = m0; mi < m1; ++mi) {
        resolve_mask<W>(c, ip, sf_idx, sf, det.masks[mi], trf, cfg, external_tol);
        if (c.is_probably_inside()) {
            return true;
        }
    }
    return false;
}

// ------------------------------------------------------- update_status
template <typename S>
DPROP_HD void update_status(nav_state<S>& nav, const nav_cfg<S>& cfg) {
    if (!nav.cache_exhausted() &&
        fabs(nav.target().path) < cfg.isect.path_tol) {
        nav.status = nav.target().is_portal() ? e_on_portal : e_on_object;
        ++nav.next;
    } else {
        nav.status = e_towards_object;
    }
    nav.trust = (nav.cache_exhausted() || nav.is_on_portal()) ? e_no_trust
                                                              : e_full_trust;
}

// ------------------------------------------------------- grid search
// Regular axis binning: int((v - min) / width + 1) - 1
template <typename S>
DPROP_HD int axis_bin(S v, S lo, S hi, uint32_t n) {
    const S width = (hi - lo) / static_cast<S>(n);
    const S u = (v - lo) / width + S(1);
    // out-of-range values (a failed reference-surface intersection) are
    // saturated instead of overflowing the integer conversion
    int b;
    if (!(u == u)) {
        b = 0;
    } else if (u >= S(2147483000)) {
        b = 2147483000;
    } else if (u <= S(-2147483000)) {
        b = -2147483000;
    } else {
        b = static_cast<int>(u);
    }
    return b - 1;
}

// Closed axis: clamp the bin window, returns [lo, hi)
DPROP_HD void closed_range(int lbin, int ubin, int bins, int& lo,
                                  int& hi) {
    int mn = lbin > 0 ? lbin : 0;
    mn = mn >= bins ? bins - 1 : mn;
    int mx = ubin >= bins ? bins - 1 : ubin;
    mx = mx < 0 ? 0 : mx;
    lo = mn;
    hi = mx + 1;
}

DPROP_HD int wrap_bin(int b, int bins) {
    return (bins + (b % bins)) % bins;
}

template <typename S, bool W>
DPROP_HD void grid_search(nav_state<S>& nav, const detector_view<S, W>& det,
                          const dev_grid<S>& g, const track_view<S>& trk,
                          vec3<S> ro, vec3<S> rd, const nav_cfg<S>& cfg,
                          const isect_cfg<S>& icfg) {
    // local position of the track on the grid's reference surface,
    // searched along the track direction (spatial_grid.hpp:100-140, 169-201)
    S p0, p1;
    if (g.kind == 1u) {
        const isect_point<S> ip = intersect_portal_cylinder(
            trk.pos, trk.dir, g.radius, -limits<S>::max());
        const vec3<S> at = trk.pos + ip.path * trk.dir;
        p0 = phi_of(at);
        p1 = ip.glob.z;
    } else {
        const dev_transform<S>& trf = det.transforms[g.transform];
        const isect_point<S> ip = intersect_plane(trk.pos, trk.dir, trf);
        const vec3<S> l = trf.point_to_local(ip.glob);
        p0 = perp(l);
        p1 = phi_of(l);
    }
    const int n0 = static_cast<int>(g.n0);
    const int n1 = static_cast<int>(g.n1);
    const int w0 = static_cast<int>(cfg.win0);
    const int w1 = static_cast<int>(cfg.win1);
    const int b0 = axis_bin(p0, g.min0, g.max0, g.n0);
    const int b1 = axis_bin(p1, g.min1, g.max1, g.n1);
    int lo0, hi0, lo1, hi1;
    if (g.kind == 1u) {
        // axis 0: phi circular, axis 1: z closed
        lo0 = b0 - w0;
        hi0 = b0 + w1 + 1;
        closed_range(b1 - w0, b1 + w1, n1, lo1, hi1);
    } else {
        // axis 0: r closed, axis 1: phi circular
        closed_range(b0 - w0, b0 + w1, n0, lo0, hi0);
        lo1 = b1 - w0;
        hi1 = b1 + w1 + 1;
    }
    for (int i0 = lo0; i0 < hi0; ++i0) {
        const int j0 = (g.kind == 1u) ? wrap_bin(i0, n0) : i0;
        for (int i1 = lo1; i1 < hi1; ++i1) {
            const int j1 = (g.kind == 1u) ? i1 : wrap_bin(i1, n1);
            const uint32_t b = g.bin_offset + static_cast<uint32_t>(j0) +
                               static_cast<uint32_t>(j1) * g.n0;
            if constexpr (W) {
                // the bin's surfaces as a range of grid_bins: [begin, end)
                // of a dynamic bin, or the bin's own entry (empty if
                // invalid); one call site keeps a single inlined copy of the
                // candidate search
                uint32_t e0 = b;
                uint32_t e1 = (det.grid_bins[b] != k_invalid) ? b + 1u : b;
                if (g.multi) {
                    e0 = det.grid_bins[b];
                    e1 = det.grid_bins[b + 1u];
                }
                for (uint32_t e = e0; e < e1; ++e) {
                    candidate_search(nav, det, det.grid_bins[e], ro, rd, icfg);
                }
            } else {
                const uint32_t sf = det.grid_bins[b];
                if (sf != k_invalid) {
                    candidate_search(nav, det, sf, ro, rd, icfg);
                }
            }
        }
    }
}

// --------------------------------------------------- local_navigation
template <typename S, bool W>
DPROP_HD_COLD void local_navigation(nav_state<S>& nav, const detector_view<S, W>& det,
                               const track_view<S>& trk, const nav_cfg<S>& cfg,
                               bool resolve_overstepping) {
    const dev_volume vol = det.volumes[nav.volume];
    nav.clear_cache();
    isect_cfg<S> icfg = cfg.isect;
    icfg.overstep_tol = resolve_overstepping ? cfg.isect.overstep_tol
                                             : -cfg.isect.path_tol;
    const vec3<S> ro = trk.pos;
    const vec3<S> rd = nav.direction * trk.dir;
    // portals and passives (brute force), then the sensitive surface grid,
    // in the order of the volume's accelerator links
    for (uint32_t i = vol.bf_begin; i < vol.bf_end; ++i) {
        candidate_search(nav, det, det.bf_surfaces[i], ro, rd, icfg);
    }
    if (vol.grid != k_invalid) {
        const dev_grid<S> g = det.grids[vol.grid];
        grid_search(nav, det, g, trk, ro, rd, cfg, icfg);
    }
    update_status(nav, cfg);
    if (nav.trust != e_full_trust) {
        if (nav.is_on_portal()) {
            nav.trust = (nav.current().volume_link == k_invalid_link)
                            ? e_full_trust
                            : e_no_trust;
        }
    }
    DPROP_NAV_TRACE(nav, "Init complete: ", trk.pos);
}

// ------------------------------------------------------- volume_switch
template <typename S, bool W>
DPROP_HD void volume_switch(nav_state<S>& nav, const detector_view<S, W>& det,
                            const track_view<S>& trk, const nav_cfg<S>& cfg) {
    if (nav.current().volume_link == k_invalid_link) {
        nav.status = e_nav_exit;
        return;
    }
    nav.set_volume(nav.current().volume_link);
    // the reference calls local_navigation with its default
    // resolve_overstepping = true here (navigation_functions.hpp:281)
    local_navigation(nav, det, trk, cfg, true);
    nav.trust = e_full_trust;
}

// ------------------------------------------------------- init_loose_cfg
template <typename S, bool W>
DPROP_HD_COLD void init_loose(nav_state<S>& nav, const detector_view<S, W>& det,
                         const track_view<S>& trk, nav_cfg<S> loose) {
    const S a = S(100) * loose.isect.overstep_tol;
    const S b = S(-10) * loose.isect.max_mask_tol;
    loose.isect.overstep_tol = a < b ? a : b;
    local_navigation(nav, det, trk, loose, true);
    if (nav.trust != e_full_trust || nav.cache_exhausted()) {
        nav.abort(e_reason_no_surface);
    }
}

// ------------------------------------------- navigator init / update
template <typename S, bool W>
DPROP_HD void navigator_init(nav_state<S>& nav, const detector_view<S, W>& det,
                             const track_view<S>& trk, const nav_cfg<S>& cfg) {
    local_navigation(nav, det, trk, cfg, false);
}

// caching_navigator::update_impl, high-trust branch: re-intersect only the
// target.  Returns true if the update is complete (update_impl returned
// there); false if trust dropped to fair and the cache must be re-evaluated.
template <typename S, bool W>
DPROP_HD bool high_trust_update(nav_state<S>& nav, const detector_view<S, W>& det,
                                const track_view<S>& trk,
                                const nav_cfg<S>& cfg) {
    const vec3<S> ro = trk.pos;
    const vec3<S> rd = nav.direction * trk.dir;
    if (!update_candidate(nav.target(), det, ro, rd, cfg.isect,
                          nav.external_tol, nav.n_isect)) {
        nav.status = e_nav_unknown;
        nav.set_fair_trust();
        return false;
    }
    update_status(nav, cfg);
    DPROP_NAV_TRACE(nav, "Update complete: high trust: ", trk.pos);
    if (nav.status == e_towards_object || nav.is_on_portal()) {
        return true;
    }
    if (nav.trust == e_full_trust &&
        update_candidate(nav.target(), det, ro, rd, cfg.isect,
                         nav.external_tol, nav.n_isect)) {
        return true;
    }
    nav.set_fair_trust();
    return false;
}

// caching_navigator::update_impl, fair- and no-trust branches.  Returns
// whether the volume was (re-)initialised.
template <typename S, bool W>
DPROP_HD_COLD bool fair_or_no_trust_update(nav_state<S>& nav,
                                           const detector_view<S, W>& det,
                                           const track_view<S>& trk,
                                           const nav_cfg<S>& cfg) {
    const vec3<S> ro = trk.pos;
    const vec3<S> rd = nav.direction * trk.dir;
    if (nav.trust == e_fair_trust && !nav.cache_exhausted()) {
        const int b = nav.begin_index();
        const int e = nav.end_index();
        for (int i = b; i < e; ++i) {
            if (!update_candidate(nav.cand[i], det, ro, rd, cfg.isect,
                                  nav.external_tol, nav.n_isect)) {
                nav.cand[i].path = limits<S>::max();
            }
        }
        // stable insertion sort of [b, e) by |path|
        for (int i = b + 1; i < e; ++i) {
            const candidate<S> key = nav.cand[i];
            const S ak = fabs(key.path);
            int j = i - 1;
            while (j >= b && fabs(nav.cand[j].path) > ak) {
                nav.cand[j + 1] = nav.cand[j];
                --j;
            }
            nav.cand[j + 1] = key;
        }
        nav.next = static_cast<int8_t>(b);
        // first unreachable candidate bounds the cache
        int inv = k_cache;
        for (int i = 0; i < k_cache; ++i) {
            if (nav.cand[i].path == limits<S>::max()) {
                inv = i;
                break;
            }
        }
        nav.last = static_cast<int8_t>(inv - 1);
        update_status(nav, cfg);
        DPROP_NAV_TRACE(nav, "Update complete: fair trust: ", trk.pos);
        if (nav.cache_exhausted()) {
            nav.set_no_trust();
        }
    }
    if (nav.trust == e_no_trust) {
        local_navigation(nav, det, trk, cfg, true);
        return true;
    }
    return false;
}

// Volume switch and loose re-initialisation after the trust-level update
// (navigator_base::update, navigator_base.hpp:121-140).
template <typename S, bool W>
DPROP_HD_COLD bool finish_update(nav_state<S>& nav, const detector_view<S, W>& det,
                                 const track_view<S>& trk,
                                 const nav_cfg<S>& cfg, bool is_init) {
    if (nav.is_on_portal()) {
        volume_switch(nav, det, trk, cfg);
        is_init = true;
        if (!nav.is_alive()) {
            return false;
        }
    }
    if (nav.trust != e_full_trust || nav.cache_exhausted()) {
        is_init = true;
        init_loose(nav, det, trk, cfg);
    }
    return is_init;
}

// navigator_base::update
template <typename S, bool W>
DPROP_HD bool navigator_update(nav_state<S>& nav, const detector_view<S, W>& det,
                               const track_view<S>& trk,
                               const nav_cfg<S>& cfg) {
    if (nav.trust == e_full_trust) {
        return false;
    }
    bool is_init = false;
    if (nav.trust == e_high_trust && high_trust_update(nav, det, trk, cfg)) {
        is_init = false;
    } else {
        is_init = fair_or_no_trust_update(nav, det, trk, cfg);
    }
    if (nav.is_on_portal() || nav.trust != e_full_trust ||
        nav.cache_exhausted()) {
        return finish_update(nav, det, trk, cfg, is_init);
    }
    return is_init;
}

}  // namespace dprop
