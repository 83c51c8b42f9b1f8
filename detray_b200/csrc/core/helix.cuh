// Helix "truth" intersections: the exact helical trajectory of a track in a
// constant field intersected with every surface of the detector by
// Newton-Raphson root finding - the reference's navigation-validation
// scanner, run on the GPU.
//
// Reference:
//   helix trajectory     core/include/detray/tracks/helix.hpp:32-180
//   root finding         core/include/detray/utils/root_finding.hpp:38-360
//                        (expand_bracket, newton_raphson_safe: Newton steps
//                        safeguarded by bisection, Numerical Recipes rtsafe)
//   helix intersectors   navigation/intersection/helix_plane_intersector.hpp
//                        :62-118, helix_cylinder_intersector.hpp:65-170,
//                        helix_line_intersector.hpp:48-150
//   mask resolution      root_finding.hpp:374-430 (resolve_mask for helix
//                        intersection points)
//   scan                 tests/include/detray/test/validation/
//                        detector_scanner.hpp:52-140 (brute_force_scan over
//                        all surfaces, kept if along the track, sorted by
//                        |path|, cut after the first world exit)
#pragma once

#include "actors.cuh"

namespace dprop {

template <typename S>
struct helix {
    vec3<S> pos0;
    vec3<S> t0;   // unit direction at s = 0
    vec3<S> h0;   // unit field direction
    vec3<S> n0;   // unit h0 x t0
    S qop;
    S B;          // field magnitude
    S alpha;      // |h0 x t0|
    S delta;      // h0 . t0
    S K;          // -q/p * B
    bool straight;  // no transverse momentum: moves along the field axis

    DPROP_HD void init(vec3<S> p, vec3<S> dir, S q_over_p, vec3<S> bfield) {
        pos0 = p;
        t0 = dir;
        qop = q_over_p;
        B = norm(bfield);
        h0 = (S(1) / B) * bfield;
        const vec3<S> hxt = cross(h0, t0);
        alpha = norm(hxt);
        n0 = (S(1) / alpha) * hxt;
        delta = dot(h0, t0);
        K = -qop * B;
        const vec3<S> mom = (S(1) / fabs(qop)) * t0;
        const S pz = dot(mom, h0);
        const vec3<S> pt = mom - pz * h0;
        straight = norm(pt) < S(1e-6);
    }
    DPROP_HD vec3<S> pos(S s) const {
        if (straight) {
            return pos0 + s * h0;
        }
        const S ks = K * s;
        const S sn = sin(ks);
        const S cs = cos(ks);
        vec3<S> r = pos0;
        r = r + (delta / K * (ks - sn)) * h0;
        r = r + (sn / K) * t0;
        r = r + (alpha / K * (S(1) - cs)) * n0;
        return r;
    }
    DPROP_HD vec3<S> dir(S s) const {
        if (straight) {
            return t0;
        }
        const S ks = K * s;
        const S cs = cos(ks);
        vec3<S> d{S(0), S(0), S(0)};
        d = d + (delta * (S(1) - cs)) * h0;
        d = d + cs * t0;
        d = d + (alpha * sin(ks)) * n0;
        return normalize(d);
    }
    // position and direction at s from one sine/cosine pair (the same
    // values as pos(s) and dir(s))
    DPROP_HD void eval(S s, vec3<S>& p, vec3<S>& d) const {
        if (straight) {
            p = pos0 + s * h0;
            d = t0;
            return;
        }
        const S ks = K * s;
        const S sn = sin(ks);
        const S cs = cos(ks);
        vec3<S> r = pos0;
        r = r + (delta / K * (ks - sn)) * h0;
        r = r + (sn / K) * t0;
        r = r + (alpha / K * (S(1) - cs)) * n0;
        p = r;
        vec3<S> v{S(0), S(0), S(0)};
        v = v + (delta * (S(1) - cs)) * h0;
        v = v + cs * t0;
        v = v + (alpha * sn) * n0;
        d = normalize(v);
    }
    DPROP_HD vec3<S> b_field() const { return B * h0; }
};

// Result of a root search: path to the root and the last step length;
// limits::max() for both when there is no root.
template <typename S>
struct root_result {
    S s;
    S ds;
};

template <typename S>
struct root_cfg {
    S tol;             // convergence: |f| or |step| below 1 um
    uint32_t max_tries;
    S max_path;        // 5 m search range
};

// Widen [a, b] (towards the side with the smaller |f|) until f changes sign;
// gives up after 1000 widenings or on non-finite values, then keeps [a, b].
template <typename S, typename F>
DPROP_HD bool expand_bracket(S a, S b, const F& f, S& lo_out, S& hi_out) {
    S lo = a > b ? b : a;
    S hi = a > b ? a : b;
    S flo = f(lo);
    S fhi = f(hi);
    uint32_t n = 0u;
    auto broken = [&]() {
        return n == 1000u || !isfinite(flo) || !isfinite(fhi) ||
               !isfinite(lo) || !isfinite(hi);
    };
    while (!signbit(flo * fhi)) {
        if (broken()) {
            lo_out = a;
            hi_out = b;
            return false;
        }
        const S w = hi - lo;
        if (fabs(flo) < fabs(fhi)) {
            lo -= w;
            flo = f(lo);
        } else {
            hi += w;
            fhi = f(hi);
        }
        ++n;
    }
    if (broken()) {
        lo_out = a;
        hi_out = b;
        return false;
    }
    lo_out = lo;
    hi_out = hi;
    return true;
}

// Safeguarded Newton-Raphson on f(s) = 0 from the guess s: bracket the
// root around s, then take Newton steps, falling back to bisection when a
// step would leave the bracket or converge slower than bisecting.  fdf(x, f,
// df) evaluates the function and its derivative.
template <typename S, typename FDF>
DPROP_HD root_result<S> newton_safe(const FDF& fdf, S s,
                                    const root_cfg<S>& cfg) {
    const S inv = limits<S>::max();
    const S eps = limits<S>::epsilon();
    const root_result<S> none{inv, inv};
    auto f_only = [&fdf](S x) {
        S fx, dfx;
        fdf(x, fx, dfx);
        return fx;
    };
    if (!(fabs(s) < inv)) {
        return none;
    }
    // initial bracket around s (the factors are single-precision constants
    // in every build, as in the reference)
    S a = (fabs(s) == S(0)) ? S(-0.2f) : S(0.8f) * s;
    S b = (fabs(s) == S(0)) ? S(0.2f) : S(1.2f) * s;
    S br0, br1;
    const bool bracketed = expand_bracket(a, b, f_only, br0, br1);
    if (bracketed) {
        s = S(0.5) * (br1 + br0);
        S fa, dfa, fb, dfb;
        fdf(br0, fa, dfa);
        fdf(br1, fb, dfb);
        if (!signbit(fa * fb) || fabs(br0) >= inv || fabs(br1) >= inv) {
            return none;
        }
        if (fabs(s) > cfg.max_path && fabs(br0) >= cfg.max_path &&
            fabs(br1) >= cfg.max_path) {
            return none;
        }
        // (the initial bracket ends are returned, as the reference does)
        if (fabs(fa) < cfg.tol) {
            return {a, eps};
        }
        if (fabs(fb) < cfg.tol) {
            return {b, eps};
        }
        // a: the end with the negative function value
        const bool lower_neg = signbit(fa);
        a = lower_neg ? br0 : br1;
        b = lower_neg ? br1 : br0;
    }
    S fs, dfs;
    fdf(s, fs, dfs);
    if (fabs(fs) < cfg.tol) {
        return {s, eps};
    }
    if (signbit(fs)) {
        a = s;
    } else {
        b = s;
    }
    S s_prev = S(0);
    uint32_t n = 0u;
    while (fabs(s - s_prev) > cfg.tol) {
        bool escapes = true;
        S s_newton = S(0);
        if (fabs(dfs) != S(0)) {
            s_newton = s - fs / dfs;
            escapes = signbit((s_newton - a) * (b - s_newton));
        }
        bool slow = true;
        const S ds_bisect = S(0.5) * (a + b) - s;
        if (bracketed && fabs(ds_bisect) < S(10) * S(unit::mm)) {
            slow = S(2) * fabs(fs) > fabs(dfs * ds_bisect + fs);
        }
        s_prev = s;
        if (bracketed && (escapes || slow || fabs(dfs) == S(0))) {
            s = S(0.5) * (a + b);
        } else {
            if (!bracketed && fabs(dfs) == S(0)) {
                return none;
            }
            s = s_newton;
        }
        fdf(s, fs, dfs);
        if (bracketed && signbit(fs)) {
            a = s;
        } else {
            b = s;
        }
        if (fabs(s) > cfg.max_path && fabs(s_prev) > cfg.max_path &&
            ((a < -cfg.max_path && b < -cfg.max_path) ||
             (a > cfg.max_path && b > cfg.max_path))) {
            return none;
        }
        ++n;
        if (n >= cfg.max_tries) {
            return none;
        }
    }
    return {s, fabs(s - s_prev)};
}

// ------------------------------------------------------------ intersectors
// Plane (rectangle, trapezoid, ring): f(s) = n . (h(s) - c)
template <typename S>
DPROP_HD root_result<S> helix_plane(const helix<S>& h,
                                    const dev_transform<S>& trf,
                                    const root_cfg<S>& cfg) {
    const vec3<S> sn = trf.z();
    const vec3<S> st = trf.translation();
    const vec3<S> dist = st - h.pos0;
    const S denom = dot(sn, h.dir(S(0.5) * norm(dist)));
    const S s_ini = (denom == S(0)) ? norm(dist) : dot(sn, dist) / denom;
    auto fdf = [&h, &sn, &st](S x, S& f, S& df) {
        vec3<S> p, d;
        h.eval(x, p, d);
        f = dot(sn, p - st);
        df = dot(sn, d);
    };
    return newton_safe(fdf, s_ini, cfg);
}

// Cylinder of radius r around the transform's z axis: f(s) =
// |(h(s) - c) x z|^2 - r^2; the two starting guesses are the ray
// intersections along the direction at half the radius.
template <typename S>
DPROP_HD void helix_cylinder(const helix<S>& h, const dev_transform<S>& trf,
                             S r, const root_cfg<S>& cfg,
                             root_result<S> out[2]) {
    const vec3<S> sz = trf.z();
    const vec3<S> sc = trf.translation();
    const vec3<S> hd = h.dir(S(0.5) * r);
    isect_point<S> ips[2];
    const int n_sol = intersect_cylinder(h.pos0, hd, trf, r, ips);
    S guess[2];
    int n_runs = n_sol;
    if (n_sol == 2) {
        guess[0] = ips[0].path;
        guess[1] = ips[1].path;
    } else if (n_sol == 1) {
        guess[0] = ips[0].path;
    } else {
        n_runs = 2;
        guess[0] = r;
        guess[1] = -r;
    }
    auto fdf = [&h, &sz, &sc, r](S x, S& f, S& df) {
        vec3<S> p, d;
        h.eval(x, p, d);
        const vec3<S> crp = cross(p - sc, sz);
        f = dot(crp, crp) - r * r;
        df = S(2) * dot(crp, cross(d, sz));
    };
    const S inv = limits<S>::max();
    out[0] = {inv, inv};
    out[1] = {inv, inv};
    for (int i = 0; i < n_runs; ++i) {
        out[i] = newton_safe(fdf, guess[i], cfg);
    }
}

// Line (wire along the transform's z axis): f(s) = t(s) . (w(s)), w the
// vector from the closest wire point to the helix point
template <typename S>
DPROP_HD root_result<S> helix_line(const helix<S>& h,
                                   const dev_transform<S>& trf,
                                   const root_cfg<S>& cfg) {
    const vec3<S> l = trf.z();
    const vec3<S> c = trf.translation();
    const vec3<S> t0 = h.dir(S(0));
    const vec3<S> r0 = h.pos(S(0));
    const S lt0 = dot(l, t0);
    const S denom = S(1) - lt0 * lt0;
    if (denom < S(1e-5)) {
        return {limits<S>::max(), limits<S>::max()};
    }
    const vec3<S> D = c - r0;
    const S P = dot(D, l);
    const S Q = dot(D, t0);
    const S s_ini = S(1) / denom * (Q - P * lt0);
    const vec3<S> bf = h.b_field();
    auto fdf = [&h, &c, &l, &bf](S x, S& f, S& df) {
        vec3<S> t, p;
        h.eval(x, p, t);
        const S A = dot(p - c, l);
        const vec3<S> w = p - (c + A * l);
        f = dot(t, w);
        const vec3<S> dtds = h.qop * cross(t, bf);
        const vec3<S> dwds = t - dot(t, l) * l;
        df = dot(dtds, w) + dot(t, dwds);
    };
    return newton_safe(fdf, s_ini, cfg);
}

// One scanned intersection
template <typename S>
struct scan_hit {
    S path;
    S loc0, loc1;
    uint32_t sf;
    uint16_t volume_link;
};

// Mask check of a helix intersection (resolve_mask for helix points):
// inside with the given tolerance, 0 on portals.
template <bool W, typename S>
DPROP_HD bool helix_inside(const dev_surface& sf, const dev_mask<S>& m,
                           const dev_transform<S>& trf, vec3<S> glob,
                           S mask_tol) {
    const S tol = (sf.kind == e_portal) ? S(0) : mask_tol;
    const vec3<S> l = trf.point_to_local(glob);
    switch (sf.shape) {
        case e_rectangle:
            return check_rectangle(m, l.x, l.y, tol, S(0)).inside;
        case e_trapezoid:
            return check_trapezoid(m, l.x, l.y, tol, S(0)).inside;
        case e_ring:
            return check_ring(m, perp(l), tol).inside;
        case e_line:
            if (W) {
                return check_line(m, l, tol, S(0)).inside;
            }
            return false;
        case e_cylinder:
        case e_concentric_cylinder:
        default:
            return check_cylinder_z(m, l.z, tol, S(0)).inside;
    }
}

// The intersections of the helix with one surface that are inside a mask
// and along the track (intersection_initialize for a helix: per mask, the
// solutions that pass it; a single-solution surface stops at the first mask
// that accepts it, a cylinder when a mask accepted both).  emit(hit) is
// called for each; the local coordinates are the surface's bound local
// coordinates at the point.
template <bool W, typename S, typename Emit>
DPROP_HD void helix_surface_hits(const detector_view<S, W>& det,
                                 uint32_t sf_idx, const helix<S>& h,
                                 S mask_tol, const root_cfg<S>& cfg,
                                 Emit&& emit) {
    const dev_surface sf = det.surfaces[sf_idx];
    const dev_transform<S>& trf = det.transforms[sf.transform];
    root_result<S> res[2];
    int n_res = 1;
    switch (sf.shape) {
        case e_cylinder:
            helix_cylinder(h, trf, det.masks[sf.mask_begin].v[0], cfg, res);
            n_res = 2;
            break;
        case e_concentric_cylinder: {
            root_result<S> two[2];
            helix_cylinder(h, trf, det.masks[sf.mask_begin].v[0], cfg, two);
            res[0] = signbit(two[0].s) ? two[1] : two[0];
            break;
        }
        case e_line:
            if (!W) {
                return;
            }
            res[0] = helix_line(h, trf, cfg);
            break;
        default:
            res[0] = helix_plane(h, trf, cfg);
    }
    // an intersection point is valid within 10 m
    bool any = false;
    for (int i = 0; i < n_res; ++i) {
        any = any || fabs(res[i].s) < S(10000) * S(unit::mm);
    }
    if (!any) {
        return;
    }
    const S inv = limits<S>::max();
    for (uint32_t mi = sf.mask_begin; mi < sf.mask_begin + sf.n_masks; ++mi) {
        const dev_mask<S> m = det.masks[mi];
        int n_found = 0;
        for (int i = 0; i < n_res; ++i) {
            const S s = res[i].s;
            if (s == inv || s == -inv) {
                continue;  // no root
            }
            const vec3<S> p = h.pos(s);
            if (!helix_inside<W>(sf, m, trf, p, mask_tol)) {
                continue;
            }
            ++n_found;
            if (!signbit(s)) {  // along the track
                const vec3<S> d = h.dir(s);
                S l0, l1;
                if (W && sf.shape == e_line) {
                    const local2<S> l = line_bound_local(trf, p, d);
                    l0 = l.l0;
                    l1 = l.l1;
                } else {
                    global_to_bound_local(sf.shape, trf, p, l0, l1);
                }
                emit(scan_hit<S>{s, l0, l1, sf_idx,
                                 static_cast<uint16_t>(m.volume_link)});
            }
            if (n_found == n_res) {
                return;
            }
        }
    }
}

// --------------------------------------------------- navigation validation
// Compare the surfaces a propagation reached (its records with
// record_all_surfaces, in path order) with the helix truth of the same track
// (navigation validation, tests/include/detray/test/validation/
// navigation_validation_utils.hpp:379-800: holes and extra surfaces).
//   - a sensitive or passive truth surface is reached if a record of the
//     same surface lies within path_tol of its path;
//   - adjacent volumes share a boundary through two coinciding portals, of
//     which the navigator records the one it continues in: a truth portal is
//     reached if any portal record lies within path_tol, and the final
//     world-exit portal if the propagation ended by leaving the world;
//   - a record is extra if no truth surface matches it the same way.
// Ti / Tr: path types of the truth and of the records.
template <typename Ti, typename Tr>
DPROP_HD void compare_trace(const uint64_t* truth_bc, const Ti* truth_path,
                            const uint16_t* truth_vlink, uint32_t n_truth,
                            const uint64_t* rec_bc, const Tr* rec_path,
                            uint32_t n_rec, bool exited, uint64_t stride,
                            uint64_t t, double path_tol, uint32_t& missed,
                            uint32_t& extra) {
    auto is_portal = [](uint64_t bc) { return ((bc >> 48) & 0xfu) == 0u; };
    missed = 0u;
    extra = 0u;
    for (uint32_t i = 0; i < n_truth; ++i) {
        const uint64_t o = static_cast<uint64_t>(i) * stride + t;
        const uint64_t bc = truth_bc[o];
        const double p = static_cast<double>(truth_path[o]);
        bool found = false;
        if (is_portal(bc) && truth_vlink[o] == k_invalid_link && exited) {
            found = true;
        }
        for (uint32_t j = 0; j < n_rec && !found; ++j) {
            const uint64_t q = static_cast<uint64_t>(j) * stride + t;
            const bool same = is_portal(bc) ? is_portal(rec_bc[q])
                                            : rec_bc[q] == bc;
            found = same &&
                    fabs(static_cast<double>(rec_path[q]) - p) <= path_tol;
        }
        missed += found ? 0u : 1u;
    }
    for (uint32_t j = 0; j < n_rec; ++j) {
        const uint64_t q = static_cast<uint64_t>(j) * stride + t;
        const uint64_t bc = rec_bc[q];
        const double p = static_cast<double>(rec_path[q]);
        bool found = false;
        for (uint32_t i = 0; i < n_truth && !found; ++i) {
            const uint64_t o = static_cast<uint64_t>(i) * stride + t;
            const bool same = is_portal(bc) ? is_portal(truth_bc[o])
                                            : truth_bc[o] == bc;
            found = same && fabs(static_cast<double>(truth_path[o]) - p) <=
                                path_tol;
        }
        extra += found ? 0u : 1u;
    }
}

}  // namespace dprop
