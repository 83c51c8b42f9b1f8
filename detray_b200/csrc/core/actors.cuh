// The actor chain run between steps: path-limit aborter, parameter
// transporter (bound -> free -> bound Jacobian and covariance transport),
// pointwise material interactor and parameter setter.
//
// Reference:
//   pathlimit_aborter            propagator/actors/aborters.hpp:23-76
//   parameter_transporter        propagator/actors/parameter_updater.hpp:314-419
//   get_full_jacobian            parameter_updater.hpp:422-572; the product
//                                F2B (P2F F2P + I) J_t B2F of
//                                codegen/detray-sympy/gen_full_jacobian.py:47-59
//   covariance transport         codegen gen_transport_covariance_to_bound_impl.py
//                                (J C J^T with the identity q/p row and time
//                                column the generator assumes)
//   frame Jacobians              propagator/detail/jacobian_{cartesian,polar,
//                                concentric_cylindrical,line}.hpp,
//                                jacobian_engine.hpp
//   parameter_setter             parameter_updater.hpp:577-627
//   external mask tolerance      propagator/detail/noise_estimation.hpp:22-107
//   material interactor          propagator/actors/pointwise_material_interactor.hpp:59-326
//   interaction formulas         material/interaction.hpp:28-310,
//                                material/detail/relativistic_quantities.hpp
//   slab / rod path segments     material/material_slab.hpp,
//                                material/material_rod.hpp
#pragma once

#include "navigator.cuh"
#include "stepper.cuh"

namespace dprop {

// index of (i, j) in the row-wise upper triangle of a symmetric 6x6 matrix
DPROP_HD constexpr int tri6(int i, int j) {
    return (i <= j) ? (i * (11 - i)) / 2 + j : (j * (11 - j)) / 2 + i;
}

// Bound track parameters of the updater state: [loc0, loc1, phi, theta,
// q/p, t], covariance, and the surface they are expressed on.
template <typename S>
struct bound_state {
    S v[6];
    S cov[21];
    uint32_t sf;  // k_invalid: no surface yet
};

template <typename S>
struct actor_cfg {
    S path_limit;
    bool use_path_limit;
    bool use_interactor;
    bool estimate_noise;
    S n_stddev;
    S accumulated_error;
    S mass;
    bool electron;  // Rossi-Greisen instead of Highland
};

// --------------------------------------------------------- local frames
template <typename S>
DPROP_HD vec3<S> bound_dir(S phi, S theta) {
    const S st = sin(theta);
    return {cos(phi) * st, sin(phi) * st, cos(theta)};
}

// The line frame's axes at a track direction (jacobian_line.hpp
// reference_frame): y along the wire, x = normalize(z x dir), z = x x y.
template <typename S>
DPROP_HD void line_frame(const dev_transform<S>& trf, vec3<S> dir,
                         vec3<S>& nx, vec3<S>& ny, vec3<S>& nz) {
    ny = trf.z();
    nx = normalize(cross(ny, dir));
    nz = cross(nx, ny);
}

// x and y axes of the line frame (the loc0 / loc1 directions)
template <typename S>
struct axes2 {
    vec3<S> x, y;
};

template <typename S>
DPROP_HD_LINE axes2<S> line_loc_axes(const dev_transform<S>& trf, vec3<S> dir) {
    axes2<S> a;
    vec3<S> nz;
    line_frame(trf, dir, a.x, a.y, nz);
    return a;
}

// line2D::local_to_global
template <typename S>
DPROP_HD_LINE vec3<S> line_to_global(const dev_transform<S>& trf, S l0, S l1,
                                     vec3<S> dir) {
    const vec3<S> on_wire = trf.point_to_global({S(0), S(0), l1});
    return on_wire + l0 * normalize(cross(trf.z(), dir));
}

// bound -> free position for the surface frame (bound_to_free_vector,
// tracks/detail/transform_track_parameters.hpp:43-74); the line frame needs
// the track direction (line2D::local_to_global)
template <typename S, bool W>
DPROP_HD vec3<S> bound_to_free_pos(const detector_view<S, W>& det,
                                   const dev_surface& sf, S l0, S l1,
                                   vec3<S> dir) {
    const dev_transform<S>& trf = det.transforms[sf.transform];
    if (W && sf.shape == e_line) {
        return line_to_global(trf, l0, l1, dir);
    }
    switch (sf.shape) {
        case e_ring:
            return trf.point_to_global({l0 * cos(l1), l0 * sin(l1), S(0)});
        case e_concentric_cylinder: {
            const S r = det.masks[sf.mask_begin].v[0];
            return {r * cos(l0), r * sin(l0), l1};
        }
        default:
            return trf.point_to_global({l0, l1, S(0)});
    }
}

// free -> bound vector on a surface (free_to_bound_vector)
template <typename S, bool W, bool Grad>
DPROP_HD void free_to_bound(const detector_view<S, W>& det, const dev_surface& sf,
                            const step_state<S, Grad>& st, S out[6]) {
    const dev_transform<S>& trf = det.transforms[sf.transform];
    if (W && sf.shape == e_line) {
        const local2<S> l = line_bound_local(trf, st.pos, st.dir);
        out[0] = l.l0;
        out[1] = l.l1;
    } else {
        global_to_bound_local(sf.shape, trf, st.pos, out[0], out[1]);
    }
    out[2] = phi_of(st.dir);
    out[3] = theta_of(st.dir);
    out[4] = st.qop;
    out[5] = st.time;
}

// columns d(pos)/d(loc0), d(pos)/d(loc1) (get_derivative_dpos_dloc)
template <typename S, bool W>
DPROP_HD void dpos_dloc(const detector_view<S, W>& det, const dev_surface& sf,
                        vec3<S> pos, vec3<S> dir, vec3<S>& c0, vec3<S>& c1) {
    const dev_transform<S>& trf = det.transforms[sf.transform];
    if (W && sf.shape == e_line) {
        const axes2<S> a = line_loc_axes(trf, dir);
        c0 = a.x;
        c1 = a.y;
        return;
    }
    switch (sf.shape) {
        case e_ring: {
            const vec3<S> l = trf.point_to_local(pos);
            const S lrad = perp(l);
            const S lphi = phi_of(l);
            const S cp = cos(lphi);
            const S sp = sin(lphi);
            const vec3<S> dx = trf.x();
            const vec3<S> dy = trf.y();
            c0 = dx * cp + dy * sp;
            c1 = (dy * cp - dx * sp) * lrad;
            return;
        }
        case e_concentric_cylinder: {
            const S r = perp(pos);
            const S ph = phi_of(pos);
            c0 = {-r * sin(ph), r * cos(ph), S(0)};
            c1 = {S(0), S(0), S(1)};
            return;
        }
        default:
            c0 = trf.x();
            c1 = trf.y();
            return;
    }
}

// rows d(loc0)/d(pos), d(loc1)/d(pos) (get_derivative_dloc_dpos)
template <typename S, bool W>
DPROP_HD void dloc_dpos(const detector_view<S, W>& det, const dev_surface& sf,
                        vec3<S> pos, vec3<S> dir, vec3<S>& r0, vec3<S>& r1) {
    const dev_transform<S>& trf = det.transforms[sf.transform];
    if (W && sf.shape == e_line) {
        const axes2<S> a = line_loc_axes(trf, dir);
        r0 = a.x;
        r1 = a.y;
        return;
    }
    switch (sf.shape) {
        case e_ring: {
            const vec3<S> l = trf.point_to_local(pos);
            const S lrad = perp(l);
            const S lphi = phi_of(l);
            const S cp = cos(lphi);
            const S sp = sin(lphi);
            const vec3<S> du = trf.x();  // first row of R^T
            const vec3<S> dv = trf.y();
            r0 = du * cp + dv * sp;
            r1 = (S(1) / lrad) * (cp * dv - sp * du);
            return;
        }
        case e_concentric_cylinder: {
            const S r_inv = S(1) / perp(pos);
            const S ph = phi_of(pos);
            r0 = {-r_inv * sin(ph), r_inv * cos(ph), S(0)};
            r1 = {S(0), S(0), S(1)};
            return;
        }
        default:
            r0 = trf.x();
            r1 = trf.y();
            return;
    }
}

// surface normal used by the path derivative and the incidence angle
template <typename S, bool W>
DPROP_HD vec3<S> surface_normal_at_pos(const detector_view<S, W>& det,
                                       const dev_surface& sf, vec3<S> pos) {
    if (sf.shape == e_concentric_cylinder) {
        const S ph = phi_of(pos);
        return {cos(ph), sin(ph), S(0)};
    }
    return det.transforms[sf.transform].z();
}

template <typename S, bool W>
DPROP_HD vec3<S> surface_normal_at_bound(const detector_view<S, W>& det,
                                         const dev_surface& sf, S l0) {
    if (sf.shape == e_concentric_cylinder) {
        return {cos(l0), sin(l0), S(0)};
    }
    return det.transforms[sf.transform].z();
}

// d(path)/d(free position), d(path)/d(free direction) to reach the surface
// (jacobian<frame>::path_derivative): -n / (n . dir) for surfaces with a
// normal; for a line (jacobian_line.hpp path_derivative) the closest
// approach also moves with the direction and the track's curvature.
template <typename S>
DPROP_HD_LINE axes2<S> line_path_derivative(const dev_transform<S>& trf,
                                            vec3<S> pos, vec3<S> dir,
                                            vec3<S> dtds) {
    const vec3<S> pc = pos - trf.translation();
    const vec3<S> z = trf.z();
    const S pz = dot(pc, z);
    const S dz = dot(z, dir);
    const vec3<S> pc_x = pc - pz * z;
    const S norm = S(-1) / (S(1) - dz * dz + dot(pc_x, dtds));
    return {norm * (dir - dz * z), norm * pc_x};
}

template <typename S, bool W>
DPROP_HD void path_derivative(const detector_view<S, W>& det,
                              const dev_surface& sf, vec3<S> pos, vec3<S> dir,
                              vec3<S> dtds, vec3<S>& f_pos, vec3<S>& f_dir) {
    if (W && sf.shape == e_line) {
        const axes2<S> f = line_path_derivative(det.transforms[sf.transform],
                                                pos, dir, dtds);
        f_pos = f.x;
        f_dir = f.y;
        return;
    }
    const vec3<S> n = surface_normal_at_pos(det, sf, pos);
    const S inv_nd = S(-1) / dot(n, dir);
    f_pos = {inv_nd * n.x, inv_nd * n.y, inv_nd * n.z};
    f_dir = {S(0), S(0), S(0)};
}

// d(pos)/d(phi), d(pos)/d(theta) of the line frame at fixed local position
// (jacobian_line.hpp get_derivative_dpos_dangle); zero for the other frames.
template <typename S>
DPROP_HD_LINE axes2<S> line_dpos_dangle(const dev_transform<S>& trf,
                                        vec3<S> pos, vec3<S> dir,
                                        vec3<S> dd_phi, vec3<S> dd_th) {
    const local2<S> l = line_bound_local(trf, pos, dir);
    vec3<S> nx, ny, nz;
    line_frame(trf, dir, nx, ny, nz);
    const S ipdn = S(1) / dot(dir, nz);
    const S C = ipdn * l.l0;
    const vec3<S> y_phi = cross(ny, dd_phi);
    const vec3<S> y_th = cross(ny, dd_th);
    return {C * (y_phi - nx * dot(nx, y_phi)), C * (y_th - nx * dot(nx, y_th))};
}

// ---------------------------------------------------- full Jacobian
// J_full (6x6) from the departure bound state, the transport Jacobian and
// the current (destination) free state.  Only rows 0..3 x cols 0..4 are
// non-trivial (the q/p row and the time column are identity, as the
// covariance-transport generator assumes); they are returned in G[4][5].
template <typename S, bool W, bool Grad>
DPROP_HD void full_jacobian(const detector_view<S, W>& det,
                            const bound_state<S>& dep, const dev_surface& dep_sf,
                            const dev_surface& dst_sf, const step_state<S, Grad>& st,
                            vec3<S> dtds, S G[4][5]) {
    // bound -> free at the departure surface
    const S ph = dep.v[2];
    const S th = dep.v[3];
    const S ct = cos(th), st_ = sin(th), cp = cos(ph), sp = sin(ph);
    const vec3<S> dep_dir{cp * st_, sp * st_, ct};
    const vec3<S> dep_pos =
        bound_to_free_pos(det, dep_sf, dep.v[0], dep.v[1], dep_dir);
    vec3<S> p0, p1;
    dpos_dloc(det, dep_sf, dep_pos, dep_dir, p0, p1);
    // ddir/dphi, ddir/dtheta
    const vec3<S> dd_phi{-st_ * sp, st_ * cp, S(0)};
    const vec3<S> dd_th{ct * cp, ct * sp, -st_};

    // M1 = J_t * B2F (8x6), rows pos(0..2), time(3), dir(4..6), qop(7)
    // pos rows: [p0 | p1 | A dd_phi | A dd_th | c | 0]
    // dir rows: [0 | 0 | B dd_phi | B dd_th | d | 0]
    // qop row:  [0 0 0 0 e 0]; time row: e5
    const transport_jac<S, Grad>& J = st.jac;
    S m1p[3][5], m1d[3][5];
    const S p0a[3] = {p0.x, p0.y, p0.z};
    const S p1a[3] = {p1.x, p1.y, p1.z};
    const S dpa[3] = {dd_phi.x, dd_phi.y, dd_phi.z};
    const S dta[3] = {dd_th.x, dd_th.y, dd_th.z};
    const S ca[3] = {J.c.x, J.c.y, J.c.z};
    const S da[3] = {J.d.x, J.d.y, J.d.z};
    for (int r = 0; r < 3; ++r) {
        S a2 = S(0), a3 = S(0), b2 = S(0), b3 = S(0);
        for (int k = 0; k < 3; ++k) {
            a2 += J.A(r, k) * dpa[k];
            a3 += J.A(r, k) * dta[k];
            b2 += J.B(r, k) * dpa[k];
            b3 += J.B(r, k) * dta[k];
        }
        m1p[r][0] = p0a[r];
        m1p[r][1] = p1a[r];
        m1p[r][2] = a2;
        m1p[r][3] = a3;
        m1p[r][4] = ca[r];
        m1d[r][0] = S(0);
        m1d[r][1] = S(0);
        m1d[r][2] = b2;
        m1d[r][3] = b3;
        m1d[r][4] = da[r];
    }
    // d(pos)/d(loc0, loc1, phi, theta) at the departure (the angle columns
    // only for the line frame), which the gradient form carries through
    // d(pos)/d(pos0) and d(dir)/d(pos0)
    S bp[3][4] = {{p0a[0], p1a[0], S(0), S(0)},
                  {p0a[1], p1a[1], S(0), S(0)},
                  {p0a[2], p1a[2], S(0), S(0)}};
    if (W && dep_sf.shape == e_line) {
        // the line frame's position also moves with the angles
        const axes2<S> cd = line_dpos_dangle(det.transforms[dep_sf.transform],
                                             dep_pos, dep_dir, dd_phi, dd_th);
        const vec3<S> c_phi = cd.x, c_th = cd.y;
        const S cpa[3] = {c_phi.x, c_phi.y, c_phi.z};
        const S cta[3] = {c_th.x, c_th.y, c_th.z};
        for (int r = 0; r < 3; ++r) {
            m1p[r][2] += cpa[r];
            m1p[r][3] += cta[r];
            bp[r][2] = cpa[r];
            bp[r][3] = cta[r];
        }
    }
    if constexpr (Grad) {
        // m1p += (P - I) bp, m1d += Q bp
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 4; ++c) {
                S a = S(0), b = S(0);
                for (int k = 0; k < 3; ++k) {
                    a += (J.P(r, k) - (r == k ? S(1) : S(0))) * bp[k][c];
                    b += J.Q(r, k) * bp[k][c];
                }
                m1p[r][c] += a;
                m1d[r][c] += b;
            }
        }
    }

    // path correction: M2 = M1 + P2F (F2P M1)
    vec3<S> f_pos, f_dir;
    path_derivative(det, dst_sf, st.pos, st.dir, dtds, f_pos, f_dir);
    const S f[3] = {f_pos.x, f_pos.y, f_pos.z};
    S s[5];
    for (int c = 0; c < 5; ++c) {
        s[c] = f[0] * m1p[0][c] + f[1] * m1p[1][c] + f[2] * m1p[2][c];
    }
    if (W && dst_sf.shape == e_line) {
        for (int c = 0; c < 5; ++c) {
            s[c] += f_dir.x * m1d[0][c] + f_dir.y * m1d[1][c] +
                    f_dir.z * m1d[2][c];
        }
    }
    const S dir_a[3] = {st.dir.x, st.dir.y, st.dir.z};
    const S dtds_a[3] = {dtds.x, dtds.y, dtds.z};
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 5; ++c) {
            m1p[r][c] += dir_a[r] * s[c];
            m1d[r][c] += dtds_a[r] * s[c];
        }
    }

    // free -> bound at the destination
    vec3<S> r0, r1;
    dloc_dpos(det, dst_sf, st.pos, st.dir, r0, r1);
    const S dth = theta_of(st.dir);
    const S dph = phi_of(st.dir);
    const S cth = cos(dth), sth = sin(dth), cph = cos(dph), sph = sin(dph);
    const S a_phi[3] = {-sph / sth, cph / sth, S(0)};
    const S a_th[3] = {cph * cth, sph * cth, -sth};
    const S r0a[3] = {r0.x, r0.y, r0.z};
    const S r1a[3] = {r1.x, r1.y, r1.z};
    for (int c = 0; c < 5; ++c) {
        G[0][c] = r0a[0] * m1p[0][c] + r0a[1] * m1p[1][c] + r0a[2] * m1p[2][c];
        G[1][c] = r1a[0] * m1p[0][c] + r1a[1] * m1p[1][c] + r1a[2] * m1p[2][c];
        G[2][c] = a_phi[0] * m1d[0][c] + a_phi[1] * m1d[1][c];
        G[3][c] = a_th[0] * m1d[0][c] + a_th[1] * m1d[1][c] +
                  a_th[2] * m1d[2][c];
    }
}

// C <- J C J^T with J = [[G (4x5), 0], [e4], [e5]]
template <typename S>
DPROP_HD void transport_covariance(const S G[4][5], S cov[21]) {
    S C[6][6];
    for (int i = 0; i < 6; ++i) {
        for (int j = 0; j < 6; ++j) {
            C[i][j] = cov[tri6(i, j)];
        }
    }
    // T = G * C[0:5, 0:6]  (4x6)
    S T[4][6];
    for (int i = 0; i < 4; ++i) {
        for (int j = 0; j < 6; ++j) {
            S a = S(0);
            for (int k = 0; k < 5; ++k) {
                a += G[i][k] * C[k][j];
            }
            T[i][j] = a;
        }
    }
    for (int i = 0; i < 4; ++i) {
        for (int j = i; j < 4; ++j) {
            S a = S(0);
            for (int k = 0; k < 5; ++k) {
                a += T[i][k] * G[j][k];
            }
            cov[tri6(i, j)] = a;
        }
        cov[tri6(i, 4)] = T[i][4];
        cov[tri6(i, 5)] = T[i][5];
    }
    // rows 4 and 5 (q/p, time) unchanged
}

// Path through a rod of radius r around a line surface at closest approach
// d (material_rod::path_segment)
template <typename S>
DPROP_HD_LINE S rod_path(S r, S cos_inc, S d) {
    if (fabs(d) > r) {
        return S(0);
    }
    const S sin_inc_2 = S(1) - cos_inc * cos_inc;
    return S(2) * sqrt((r * r - d * d) / sin_inc_2);
}

// The material slab a track at bound local (l0, l1) sees on a surface:
// its homogeneous slab or rod, or the bin of its material map that holds the
// local position (material_accessor::get, material/detail/
// material_accessor.hpp; axis binning of utils/grid/detail/axis_binning.hpp
// and the closed / circular bounds of axis_bounds.hpp)
template <typename S, bool W>
DPROP_HD dev_slab<S> surface_material(const detector_view<S, W>& det,
                                      const dev_surface& sf, S l0, S l1) {
    if (W && sf.material_map) {
        const dev_grid<S> g = det.grids[sf.material];
        const int n0 = static_cast<int>(g.n0);
        const int n1 = static_cast<int>(g.n1);
        int b0 = axis_bin(l0, g.min0, g.max0, g.n0);
        int b1 = axis_bin(l1, g.min1, g.max1, g.n1);
        // circular axes wrap, closed axes clamp (axis_bounds.hpp)
        if (g.kind == 3u) {  // (r*phi circular, z closed)
            b0 = wrap_bin(b0, n0);
        } else {
            b0 = b0 <= 0 ? 0 : (b0 >= n0 ? n0 - 1 : b0);
        }
        if (g.kind == 4u) {  // (r closed, phi circular)
            b1 = wrap_bin(b1, n1);
        } else {
            b1 = b1 <= 0 ? 0 : (b1 >= n1 ? n1 - 1 : b1);
        }
        const uint32_t slab = det.grid_bins[g.bin_offset + static_cast<uint32_t>(b0) +
                                            static_cast<uint32_t>(b1) * g.n0];
        return det.slabs[slab];
    }
    return det.slabs[sf.material];
}

// pointwise_material_interactor::update on the bound state
template <typename S, bool W>
DPROP_HD bool interact(const detector_view<S, W>& det, const dev_surface& sf,
                       bound_state<S>& b, const actor_cfg<S>& cfg, S q,
                       S nav_dir) {
    if (sf.material == k_invalid) {
        return false;
    }
    const dev_slab<S> mat = surface_material(det, sf, b.v[0], b.v[1]);
    const vec3<S> dir = bound_dir(b.v[2], b.v[3]);
    const vec3<S> n = surface_normal_at_bound(det, sf, b.v[0]);
    const S cos_inc = fabs(dot(dir, n));
    if (mat.thickness <= limits<S>::epsilon()) {
        return false;
    }
    const S qop = b.v[4];
    if (qop == S(0)) {
        return false;
    }
    S path_segment, x_over_x0;
    if (W && mat.is_rod != S(0)) {
        path_segment = rod_path(mat.thickness, cos_inc, b.v[0]);
        x_over_x0 = path_segment / mat.X0;
    } else {
        path_segment = mat.thickness / cos_inc;
        x_over_x0 = mat.thickness_in_X0 / cos_inc;
    }
    const rel_quantities<S> rq = make_rq(cfg.mass, qop, q);
    const S e_loss = path_segment * bethe_bloch(mat, rq);
    const S sigma_qop = landau_sigma_qop(path_segment, mat, rq, q);
    const S theta0 = scattering_theta0(x_over_x0, rq, q, cfg.electron);
    // energy loss
    const S m = cfg.mass;
    const S p = q / qop;
    const S next_e = sqrt(m * m + p * p) - copysign(e_loss, nav_dir);
    const S next_p = (m < next_e) ? sqrt(next_e * next_e - m * m) : S(0);
    const S next_qop = (q != S(0)) ? q / next_p : S(1) / next_p;
    b.v[4] = (next_p == S(0)) ? limits<S>::max() : next_qop;
    b.cov[tri6(4, 4)] += sigma_qop * sigma_qop;
    // multiple scattering (uses the unmodified direction)
    const S var = theta0 * theta0;
    b.cov[tri6(2, 2)] += (dir.z == S(1)) ? limits<S>::max()
                                         : var / (S(1) - dir.z * dir.z);
    b.cov[tri6(3, 3)] += var;
    return true;
}

// estimate_external_mask_tolerance (noise_estimation.hpp:22-107)
template <typename S, bool Grad>
DPROP_HD void estimate_external_tol(nav_state<S>& nav, const bound_state<S>& b,
                                    const step_state<S, Grad>& st,
                                    const actor_cfg<S>& cfg, S q) {
    const S n = cfg.n_stddev;
    const S var0 = b.cov[tri6(0, 0)];
    const S var1 = b.cov[tri6(1, 1)];
    const S dphi = n * sqrt(b.cov[tri6(2, 2)]);
    const S dth = n * sqrt(b.cov[tri6(3, 3)]);
    const S phi_err = b.v[2] + dphi;
    const S th_err = b.v[3] + dth;
    const S ste = sin(th_err);
    vec3<S> displ{cos(phi_err) * ste, sin(phi_err) * ste, cos(th_err)};
    const S max_tol = S(5);
    const S path = nav.cache_exhausted() ? max_tol : fabs(nav.target().path);
    displ = path * (displ - st.dir);
    const S p = q / st.qop;
    const S noise = S(1) / p * cfg.accumulated_error *
                    static_cast<S>(st.path_length);
    const S ext = sqrt(n * n * (var0 + var1) + dot(displ, displ) + noise * noise);
    nav.external_tol = ext > max_tol ? max_tol : ext;
}

}  // namespace dprop
