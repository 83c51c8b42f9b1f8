// Surface geometry on the propagation path: local frames, mask checks and
// ray intersections, and the navigation candidate they produce.
//
// Reference semantics followed here:
//   ray-plane        navigation/intersection/ray_plane_intersector.hpp:60-93
//   ray-cylinder     navigation/intersection/ray_cylinder_intersector.hpp:61-122
//   ray-portal cyl.  navigation/intersection/ray_cylinder_portal_intersector.hpp:67-132
//   ray-line         navigation/intersection/ray_line_intersector.hpp:58-99
//   quadratic        utils/quadratic_equation.hpp:30-90
//   resolve_mask     navigation/intersection/intersector_base.hpp:167-252
//   mask checks      geometry/shapes/{rectangle2D,trapezoid2D,ring2D,
//                    cylinder2D,concentric_cylinder2D,line}.hpp
//   local frames     geometry/coordinates/{cartesian2D,polar2D,
//                    concentric_cylindrical2D,cylindrical2D,line2D}.hpp
#pragma once

#include "tables.cuh"

namespace dprop {

enum isect_status : uint8_t { e_inside = 0, e_edge = 1, e_outside = 2 };

// A navigation candidate: intersection2D without the local position
// (navigation/intersection/intersection.hpp:188-430), 12 bytes in fp32.
template <typename S>
struct candidate {
    S path;
    uint32_t sf;           // surface index, k_invalid = no surface
    uint16_t volume_link;  // next volume, k_invalid_link = leaves the world
    uint8_t status;        // isect_status
    uint8_t flags;         // bit0: path >= 0 (along), bit1: portal surface

    DPROP_HD bool is_inside() const { return status == e_inside; }
    DPROP_HD bool is_edge() const { return status == e_edge; }
    DPROP_HD bool is_probably_inside() const { return status <= e_edge; }
    DPROP_HD bool is_portal() const { return (flags & 2u) != 0u; }
};

template <typename S>
DPROP_HD candidate<S> invalid_candidate() {
    candidate<S> c;
    c.path = limits<S>::max();
    c.sf = k_invalid;
    c.volume_link = static_cast<uint16_t>(k_invalid_link);
    c.status = e_outside;
    c.flags = 1u;
    return c;
}

// Navigation tolerances (intersection::config, intersection_config.hpp:20-33)
template <typename S>
struct isect_cfg {
    S min_mask_tol;
    S max_mask_tol;
    S mask_tol_scalor;
    S path_tol;
    S overstep_tol;
    bool min_tol_is_max;  // min_mask_tolerance == FLT_MAX (forces tolerances)
};

// Intersection point of a ray with a surface (intersection_point with
// position).  For portal cylinders only z is known (point_type = 2D).
template <typename S>
struct isect_point {
    S path;
    vec3<S> glob;
};

template <typename S>
DPROP_HD bool ip_valid(S path) {
    // intersection_point::is_valid: |path| < 10 m (intersection.hpp:53-56)
    return fabs(path) < S(10000);
}

// ---------------------------------------------------------------- masks
// Returns (precise, with_edge) like check_boundaries; shapes whose check
// ignores the edge tolerance return precise for both.
template <typename S>
struct mask_result {
    bool inside;
    bool edge;
};

template <typename S>
DPROP_HD mask_result<S> check_rectangle(const dev_mask<S>& m, S l0, S l1,
                                        S tol, S edge_tol) {
    const S a0 = fabs(l0);
    const S a1 = fabs(l1);
    mask_result<S> r;
    r.inside = (a0 <= m.v[0] + tol) && (a1 <= m.v[1] + tol);
    r.edge = false;
    if (edge_tol > S(0)) {
        const S ft = tol + edge_tol;
        r.edge = (a0 <= m.v[0] + ft) && (a1 <= m.v[1] + ft);
    }
    return r;
}

template <typename S>
DPROP_HD mask_result<S> check_trapezoid(const dev_mask<S>& m, S l0, S l1,
                                        S tol, S edge_tol) {
    const S rel_y = (m.v[2] + l1) * m.v[3];
    const S bound_x = m.v[0] + rel_y * (m.v[1] - m.v[0]);
    mask_result<S> r;
    r.inside = (fabs(l0) <= bound_x + tol) && (fabs(l1) <= m.v[2] + tol);
    r.edge = false;
    if (edge_tol > S(0)) {
        const S ft = tol + edge_tol;
        r.edge = (fabs(l0) <= bound_x + ft) && (fabs(l1) <= m.v[2] + ft);
    }
    return r;
}

template <typename S>
DPROP_HD mask_result<S> check_ring(const dev_mask<S>& m, S r, S tol) {
    const bool in = (r + tol >= m.v[0]) && (r <= m.v[1] + tol);
    return {in, in};
}

template <typename S>
DPROP_HD mask_result<S> check_cylinder_z(const dev_mask<S>& m, S z, S tol,
                                         S edge_tol) {
    mask_result<S> r;
    r.inside = (m.v[1] - tol <= z) && (z <= m.v[2] + tol);
    r.edge = false;
    if (edge_tol > S(0)) {
        const S ft = tol + edge_tol;
        r.edge = (m.v[1] - ft <= z) && (z <= m.v[2] + ft);
    }
    return r;
}

template <typename S>
DPROP_HD mask_result<S> check_portal_z(const dev_mask<S>& m, S z, S tol) {
    const bool in = (m.v[1] - tol <= z) && (z <= m.v[2] + tol);
    return {in, in};
}

// line<square>: a drift cell, |x|, |y| <= half width, |z| <= half_z in the
// cartesian frame of the wire; line<circular>: a straw tube,
// radius <= r, |z| <= half_z (line.hpp check_boundaries)
template <typename S>
DPROP_HD_LINE mask_result<S> check_line(const dev_mask<S>& m, vec3<S> l, S tol,
                                        S edge_tol) {
    mask_result<S> r;
    r.edge = false;
    if (m.v[2] != S(0)) {
        const S a0 = fabs(l.x), a1 = fabs(l.y), a2 = fabs(l.z);
        r.inside = a0 <= (m.v[0] + tol) && a1 <= (m.v[0] + tol) &&
                   a2 <= (m.v[1] + tol);
        if (edge_tol > S(0)) {
            const S ft = tol + edge_tol;
            r.edge = a0 <= (m.v[0] + ft) && a1 <= (m.v[0] + ft) &&
                     a2 <= (m.v[1] + ft);
        }
        return r;
    }
    const S a0 = fabs(perp(l));
    const S a1 = fabs(l.z);
    r.inside = a0 <= (m.v[0] + tol) && a1 <= (m.v[1] + tol);
    if (edge_tol > S(0)) {
        const S ft = tol + edge_tol;
        r.edge = a0 <= (m.v[0] + ft) && a1 <= (m.v[1] + ft);
    }
    return r;
}

// Mask check of a global intersection point, resolving the local frame of
// the shape (mask::resolve, geometry/mask.hpp).
// W: the detector may hold line surfaces
template <bool W, typename S>
DPROP_HD mask_result<S> check_mask(uint8_t shape, const dev_mask<S>& m,
                                   const dev_transform<S>& trf,
                                   const isect_point<S>& ip, S tol,
                                   S edge_tol) {
    switch (shape) {
        case e_rectangle: {
            const vec3<S> l = trf.point_to_local(ip.glob);
            return check_rectangle(m, l.x, l.y, tol, edge_tol);
        }
        case e_trapezoid: {
            const vec3<S> l = trf.point_to_local(ip.glob);
            return check_trapezoid(m, l.x, l.y, tol, edge_tol);
        }
        case e_ring: {
            const vec3<S> l = trf.point_to_local(ip.glob);
            return check_ring(m, perp(l), tol);
        }
        case e_cylinder: {
            const vec3<S> l = trf.point_to_local(ip.glob);
            return check_cylinder_z(m, l.z, tol, edge_tol);
        }
        case e_line:
            if (W) {
                return check_line(m, trf.point_to_local(ip.glob), tol,
                                  edge_tol);
            }
            return {false, false};
        case e_concentric_cylinder:
        default: {
            // the portal intersector only provides the global z
            return check_portal_z(m, ip.glob.z, tol);
        }
    }
}

// resolve_mask (intersector_base.hpp:167-252) for one mask of a surface
template <bool W, typename S>
DPROP_HD void resolve_mask(candidate<S>& is, const isect_point<S>& ip,
                           uint32_t sf_idx, const dev_surface& sf,
                           const dev_mask<S>& m, const dev_transform<S>& trf,
                           const isect_cfg<S>& cfg, S external_tol) {
    is.status = e_outside;
    if (!(ip.path >= cfg.overstep_tol)) {
        return;
    }
    S base_tol = S(0);
    S ext_tol = S(0);
    if (sf.kind != e_portal || cfg.min_tol_is_max) {
        ext_tol = external_tol;
        base_tol = max_(cfg.min_mask_tol,
                        min_(cfg.max_mask_tol, cfg.mask_tol_scalor * fabs(ip.path)));
    }
    const mask_result<S> r =
        check_mask<W>(sf.shape, m, trf, ip, base_tol, ext_tol);
    if (r.edge) {
        is.status = e_edge;
    }
    if (r.inside) {
        is.status = e_inside;
    }
    is.path = ip.path;
    is.sf = sf_idx;
    is.flags = static_cast<uint8_t>((signbit(ip.path) ? 0u : 1u) |
                                    (sf.kind == e_portal ? 2u : 0u));
    is.volume_link = static_cast<uint16_t>(m.volume_link);
}

// --------------------------------------------------------- intersectors
// Stable roots of a x^2 + b x + c (quadratic_equation.hpp:30-90).
template <typename S>
DPROP_HD int solve_quadratic(S a, S b, S c, S& s0, S& s1) {
    const S tol = limits<S>::epsilon();
    s0 = limits<S>::max();
    s1 = limits<S>::max();
    if (fabs(a) <= tol) {
        if (fabs(b) <= tol) {
            return 0;
        }
        s0 = -c / b;
        return 1;
    }
    const S discr = b * b - S(4) * a * c;
    if (discr > tol) {
        const S q = S(-0.5) * (b + copysign(sqrt(discr), b));
        S v0 = q / a;
        S v1 = c / q;
        if (v0 > v1) {
            const S t = v0;
            v0 = v1;
            v1 = t;
        }
        s0 = v0;
        s1 = v1;
        return 2;
    }
    if (discr >= S(0)) {
        s0 = S(-0.5) * b / a;
        return 1;
    }
    return 0;
}

// Plane (rectangle, trapezoid, ring): ray_plane_intersector.hpp:60-87
template <typename S>
DPROP_HD isect_point<S> intersect_plane(vec3<S> ro, vec3<S> rd,
                                        const dev_transform<S>& trf) {
    isect_point<S> ip;
    const vec3<S> sn = trf.z();
    const S denom = dot(rd, sn);
    if (denom == S(0)) {
        ip.path = limits<S>::max();
        ip.glob = {limits<S>::max(), limits<S>::max(), limits<S>::max()};
        return ip;
    }
    ip.path = dot(sn, trf.translation() - ro) / denom;
    ip.glob = ro + ip.path * rd;
    return ip;
}

// Concentric (portal / beampipe) cylinder around z:
// ray_cylinder_portal_intersector.hpp:67-132.  The radial difference is
// formed in S and widened to double exactly as the reference does; the
// discriminant is then evaluated in double before narrowing.
template <typename S>
DPROP_HD isect_point<S> intersect_portal_cylinder(vec3<S> ro, vec3<S> rd,
                                                  S r, S overstep_tol) {
    isect_point<S> ip;
    const S inv = limits<S>::max();
    ip.path = inv;
    ip.glob = {inv, inv, inv};
    const S rd_perp_2 = rd.x * rd.x + rd.y * rd.y;
    if (rd_perp_2 < limits<S>::epsilon()) {
        return ip;
    }
    const S ro_perp_2 = ro.x * ro.x + ro.y * ro.y;
    S path = inv;
    const double rad_diff = static_cast<double>(r * r - ro_perp_2);
    if (fabs(rad_diff) > 1e-3) {
        const S rd_perp_inv_2 = S(1) / rd_perp_2;
        const S k = -rd_perp_inv_2 * (ro.x * rd.x + ro.y * rd.y);
        const S discr = static_cast<S>(static_cast<double>(rd_perp_inv_2) *
                                           rad_diff +
                                       static_cast<double>(k * k));
        if (discr < S(0)) {
            return ip;
        }
        const S sq = sqrt(discr);
        const S s1 = k + sq;
        const S s2 = k - sq;
        path = (fabs(s1) < fabs(s2)) ? s1 : s2;
        if (path < overstep_tol && sq > S(0)) {
            path = (fabs(s1) >= fabs(s2)) ? s1 : s2;
        }
    } else {
        path = static_cast<S>(rad_diff);
    }
    if (path < overstep_tol) {
        path = inv;
    }
    ip.path = path;
    ip.glob = {inv, inv, ro.z + path * rd.z};
    return ip;
}

// General cylinder (cylinder2D): ray_cylinder_intersector.hpp:61-122,
// two solutions ordered by path.
template <typename S>
DPROP_HD int intersect_cylinder(vec3<S> ro, vec3<S> rd,
                                const dev_transform<S>& trf, S r,
                                isect_point<S> out[2]) {
    const vec3<S> sz = trf.z();
    const vec3<S> sc = trf.translation();
    const vec3<S> pc_cross_sz = cross(ro - sc, sz);
    const vec3<S> rd_cross_sz = cross(rd, sz);
    const S a = dot(rd_cross_sz, rd_cross_sz);
    const S b = S(2) * dot(rd_cross_sz, pc_cross_sz);
    const S c = dot(pc_cross_sz, pc_cross_sz) - r * r;
    S s0, s1;
    const int n = solve_quadratic(a, b, c, s0, s1);
    const S inv = limits<S>::max();
    out[0].path = inv;
    out[1].path = inv;
    out[0].glob = out[1].glob = {inv, inv, inv};
    if (n == 2) {
        out[1].path = s1;
        out[1].glob = ro + s1 * rd;
    }
    if (n >= 1) {
        out[0].path = s0;
        out[0].glob = ro + s0 * rd;
    }
    return n;
}

// Line (wire): the point of closest approach of the ray to the wire,
// ray_line_intersector.hpp:58-99.  A ray (almost) parallel to the wire has
// no intersection.
template <typename S>
DPROP_HD_LINE isect_point<S> intersect_line(vec3<S> ro, vec3<S> rd,
                                            const dev_transform<S>& trf) {
    isect_point<S> ip;
    const vec3<S> z = trf.z();
    const S zd = dot(z, rd);
    const S denom = S(1) - zd * zd;
    if (denom < S(1e-5)) {
        ip.path = limits<S>::max();
        ip.glob = {limits<S>::max(), limits<S>::max(), limits<S>::max()};
        return ip;
    }
    const vec3<S> t2l = trf.translation() - ro;
    const S t2l_on_line = dot(t2l, z);
    const S t2l_on_track = dot(t2l, rd);
    ip.path = S(1) / denom * (t2l_on_track - t2l_on_line * zd);
    ip.glob = ro + ip.path * rd;
    return ip;
}

// ----------------------------------------------- local frames (bound loc)
// line2D (geometry/coordinates/line2D.hpp): loc0 = signed distance from the
// wire, negative when the wire lies on the side of z x dir; loc1 = position
// along the wire.
template <typename S>
struct local2 {
    S l0, l1;
};

template <typename S>
DPROP_HD_LINE local2<S> line_bound_local(const dev_transform<S>& trf,
                                         vec3<S> p, vec3<S> dir) {
    const vec3<S> local3 = trf.point_to_local(p);
    const vec3<S> r = cross(trf.z(), dir);
    const S sign = dot(r, trf.translation() - p) > S(0) ? S(-1) : S(1);
    return {sign * perp(local3), local3.z};
}

// free_to_bound: the two local coordinates of a global point on the surface
template <typename S>
DPROP_HD void global_to_bound_local(uint8_t shape,
                                    const dev_transform<S>& trf, vec3<S> p,
                                    S& l0, S& l1) {
    switch (shape) {
        case e_ring: {  // polar2D
            const vec3<S> l = trf.point_to_local(p);
            l0 = perp(l);
            l1 = phi_of(l);
            return;
        }
        case e_concentric_cylinder: {  // concentric_cylindrical2D
            l0 = phi_of(p);
            l1 = p.z;
            return;
        }
        case e_cylinder: {  // cylindrical2D: (r * phi, z) in the local frame
            const vec3<S> l = trf.point_to_local(p);
            l0 = perp(l) * phi_of(l);
            l1 = l.z;
            return;
        }
        case e_rectangle:
        case e_trapezoid:
        default: {  // cartesian2D
            const vec3<S> l = trf.point_to_local(p);
            l0 = l.x;
            l1 = l.y;
            return;
        }
    }
}

}  // namespace dprop
