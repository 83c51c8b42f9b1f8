// Reverse-mode derivatives of the recorded bound parameters.
//
// A propagation records, at every transported surface k (sensitive, or
// carrying material), the bound parameters b_k = (loc0, loc1, phi, theta,
// q/p, t) after the material interaction.  For a loss L(b_1 .. b_K) given by
// its gradients g_k = dL/db_k, this file computes
//   dL/d(initial free parameters x, y, z, t, tx, ty, tz, q/p)
//   dL/d(alignment of every planar or ring surface a record lies on)
// by one reverse sweep over the records of each track.
//
// Chain of one track (the forward pass in adjoint mode writes the tape):
//   b_1^- = T_1(x0)            start -> first surface, Jacobian K (5 x 7)
//   b_k^+ = M_k(b_k^-)         material kick: only q/p changes
//   b_k^- = T_k(b_{k-1}^+)     surface to surface, Jacobian J_k
// J_k = F2B (P2F F2P + I) J_transport B2F is the full Jacobian the reference's
// parameter transporter forms for its covariance transport
// (propagator/actors/parameter_updater.hpp:422-572,
// codegen gen_full_jacobian.py:47-59); its non-trivial 4 x 5 block G_k is on
// the tape, the q/p row and the time column are identity (the reference's
// convention, which also leaves the time row as identity: time derivatives
// pass straight through).  Unlike the reference's covariance path, adjoint
// mode restarts the transport Jacobian at the first transported surface too,
// so that J_2 is the derivative of the step chain from surface 1 (the
// reference keeps integrating from the track start there).
//
// Reverse sweep, a_k = dL/db_k^+ and c_k = dL/db_k^-:
//   a_K = g_K;  a_k = g_k + J_{k+1}^T c_{k+1};  c_k = M_k^T a_k
//   dL/dx0 = K^T c_1
// M_k is identity but for its q/p row dq+/d(loc0, phi, theta, q/p), formed
// from dq+/dq- and dq+/d(d.n) on the tape (the energy loss depends on q/p
// and on the incidence d.n; pointwise_material_interactor.hpp:59-326,
// material/interaction.hpp:28-150).
//
// Alignment of surface s (record k): translation dt and small rotation w
// about the surface centre c, in global axes.  First order, with u, v, n the
// local axes, x the intersection, r = x - c, d the direction:
//   ds          = (n.dt - w.(n x r)) / (n.d)        the intersection moves
//   dloc_u      = w.(u x r) + (u.d) ds - u.dt       (same for v)
//   d(dir)      = dtds^- ds                          incoming curvature
//   d(d.n)      = (dtds^-.n) ds + w.(n x d)          incidence -> q/p kick
// (ring surfaces chain dloc through their polar coordinates).  The surface
// also moves the point where the material kick happens; continuing from the
// moved point is the same as continuing from the old one with the direction
// changed by (dtds^- - dtds^+) ds = (1 - q+/q-) dtds^- ds and the new q/p.
// So the alignment derivative is
//   dL/d(delta) = g_k . db_k^+/d(delta) + (a_k - g_k) . db~/d(delta)
// with db~ = (0, 0, that direction change, d(q+), 0).  Step sizes and the
// navigation's choices are constants of the derivative (discrete adjoint of
// the adaptive integration); the transport Jacobian does not differentiate
// the field map (no field gradient, as in the reference).
#pragma once

#include "actors.cuh"

namespace dprop {

// Per-record tape components, each a [capacity][n] slot-major plane.
enum tape_component : int {
    e_tape_g = 0,          // G row-major, 20 values
    e_tape_mq = 20,        // d(q/p)+ / d(q/p)-
    e_tape_mc = 21,        // d(q/p)+ / d(d.n)
    e_tape_dtds = 22,      // dtds before the kick, 3 values
    e_tape_qop_in = 25,    // q/p before the kick
    e_tape_repeat = 26,    // 1: record repeats the previous surface (no transport)
    k_tape_rec = 27,
};
// Per-track tape: K row-major (rows loc0, loc1, phi, theta, q/p; columns
// x, y, z, tx, ty, tz, q/p), one [n] plane each.
constexpr int k_tape_init = 35;

template <typename S>
struct tape_view {
    S* rec;
    S* init;
    uint64_t n;
    uint32_t capacity;

    DPROP_HD S& r(int c, uint32_t k, uint64_t t) const {
        return rec[(static_cast<uint64_t>(c) * capacity + k) * n + t];
    }
    DPROP_HD S& i(int c, uint64_t t) const {
        return init[static_cast<uint64_t>(c) * n + t];
    }
};

// Forward-side writer handed to propagate_track in adjoint mode.
template <typename S>
struct adjoint_tape {
    static constexpr bool enabled = true;
    tape_view<S> v;
    uint64_t track;

    DPROP_HD void write_init(const S K[5][7]) const {
        for (int r = 0; r < 5; ++r) {
            for (int c = 0; c < 7; ++c) {
                v.i(r * 7 + c, track) = K[r][c];
            }
        }
    }
    DPROP_HD void write_record(uint32_t slot, const S G[4][5], S mq, S mc,
                               vec3<S> dtds, S qop_in, bool repeat) const {
        if (slot >= v.capacity) {
            return;
        }
        for (int r = 0; r < 4; ++r) {
            for (int c = 0; c < 5; ++c) {
                v.r(e_tape_g + r * 5 + c, slot, track) = G[r][c];
            }
        }
        v.r(e_tape_mq, slot, track) = mq;
        v.r(e_tape_mc, slot, track) = mc;
        v.r(e_tape_dtds + 0, slot, track) = dtds.x;
        v.r(e_tape_dtds + 1, slot, track) = dtds.y;
        v.r(e_tape_dtds + 2, slot, track) = dtds.z;
        v.r(e_tape_qop_in, slot, track) = qop_in;
        v.r(e_tape_repeat, slot, track) = repeat ? S(1) : S(0);
    }
};

// The propagation without a tape.
struct no_tape {
    static constexpr bool enabled = false;
};

// K: derivative of the bound parameters at the first transported surface
// with respect to the initial free parameters (x, y, z, tx, ty, tz, q/p),
// from the transport Jacobian accumulated since the start.  Same product as
// full_jacobian, with B2F replaced by the identity on the free parameters.
template <typename S, bool W, bool Grad>
DPROP_HD void initial_jacobian(const detector_view<S, W>& det,
                               const dev_surface& dst_sf,
                               const step_state<S, Grad>& st, vec3<S> dtds,
                               S K[5][7]) {
    const transport_jac<S, Grad>& J = st.jac;
    // M1 = J_t restricted to the columns pos (identity, or P and Q with the
    // field gradient), dir (A, B), q/p
    S mp[3][7], md[3][7];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            if constexpr (Grad) {
                mp[r][c] = J.P(r, c);
                md[r][c] = J.Q(r, c);
            } else {
                mp[r][c] = (r == c) ? S(1) : S(0);
                md[r][c] = S(0);
            }
            mp[r][3 + c] = J.A(r, c);
            md[r][3 + c] = J.B(r, c);
        }
    }
    mp[0][6] = J.c.x;
    mp[1][6] = J.c.y;
    mp[2][6] = J.c.z;
    md[0][6] = J.d.x;
    md[1][6] = J.d.y;
    md[2][6] = J.d.z;
    // path correction onto the destination surface
    vec3<S> f_pos, f_dir;
    path_derivative(det, dst_sf, st.pos, st.dir, dtds, f_pos, f_dir);
    const S dir_a[3] = {st.dir.x, st.dir.y, st.dir.z};
    const S dtds_a[3] = {dtds.x, dtds.y, dtds.z};
    for (int c = 0; c < 7; ++c) {
        const S s = f_pos.x * mp[0][c] + f_pos.y * mp[1][c] +
                    f_pos.z * mp[2][c] + f_dir.x * md[0][c] +
                    f_dir.y * md[1][c] + f_dir.z * md[2][c];
        for (int r = 0; r < 3; ++r) {
            mp[r][c] += dir_a[r] * s;
            md[r][c] += dtds_a[r] * s;
        }
    }
    // free -> bound at the destination
    vec3<S> r0, r1;
    dloc_dpos(det, dst_sf, st.pos, st.dir, r0, r1);
    const S th = theta_of(st.dir);
    const S ph = phi_of(st.dir);
    const S cth = cos(th), sth = sin(th), cph = cos(ph), sph = sin(ph);
    const S a_phi[3] = {-sph / sth, cph / sth, S(0)};
    const S a_th[3] = {cph * cth, sph * cth, -sth};
    const S r0a[3] = {r0.x, r0.y, r0.z};
    const S r1a[3] = {r1.x, r1.y, r1.z};
    for (int c = 0; c < 7; ++c) {
        K[0][c] = r0a[0] * mp[0][c] + r0a[1] * mp[1][c] + r0a[2] * mp[2][c];
        K[1][c] = r1a[0] * mp[0][c] + r1a[1] * mp[1][c] + r1a[2] * mp[2][c];
        K[2][c] = a_phi[0] * md[0][c] + a_phi[1] * md[1][c];
        K[3][c] = a_th[0] * md[0][c] + a_th[1] * md[1][c] + a_th[2] * md[2][c];
        K[4][c] = (c == 6) ? J.e : S(0);
    }
}

// Derivatives of the q/p after the kick of interact() with respect to the
// q/p before it (mq) and to the incidence d.n (mc), for the bound state b
// before the kick.  (1, 0) where interact() leaves q/p alone; (0, 0) where
// the particle stops (q/p becomes the invalid maximum).  For a material rod
// around a wire the dependence of the path on the closest approach (loc0)
// is not included.
template <typename S, bool W>
DPROP_HD void kick_derivatives(const detector_view<S, W>& det,
                               const dev_surface& sf, const S* b, S mass, S q,
                               S nav_dir, S& mq, S& mc) {
    mq = S(1);
    mc = S(0);
    if (sf.material == k_invalid) {
        return;
    }
    const dev_slab<S> mat = surface_material(det, sf, b[0], b[1]);
    const S qop = b[4];
    if (mat.thickness <= limits<S>::epsilon() || qop == S(0)) {
        return;
    }
    const vec3<S> dir = bound_dir(b[2], b[3]);
    const vec3<S> n = surface_normal_at_bound(det, sf, b[0]);
    const S dn = dot(dir, n);
    const S cos_inc = fabs(dn);
    // path through the material and its derivative by |d.n| (the closest
    // approach of a rod is held fixed)
    S path, dpath_dcos;
    if (W && mat.is_rod != S(0)) {
        path = rod_path(mat.thickness, cos_inc, b[0]);
        dpath_dcos = path * cos_inc / (S(1) - cos_inc * cos_inc);
    } else {
        path = mat.thickness / cos_inc;
        dpath_dcos = -path / cos_inc;
    }
    const rel_quantities<S> rq = make_rq(mass, qop, q);
    const S bb = bethe_bloch(mat, rq);
    const S dbb = bethe_bloch_dqop(mat, rq, bb);
    const S sgn = (nav_dir < S(0)) ? S(-1) : S(1);
    const S p = q / qop;
    const S E = sqrt(mass * mass + p * p);
    const S e1 = E - sgn * path * bb;
    if (!(mass < e1)) {
        mq = S(0);
        return;
    }
    const S p1 = sqrt(e1 * e1 - mass * mass);
    // q+ = q / p1,  dq+/de1 = -q / p1^2 * e1 / p1
    const S dq_de1 = -q / (p1 * p1) * (e1 / p1);
    // dE/dq = (p / E) dp/dq with dp/dq = -p^2 / q
    const S de1_dq = (p / E) * (-p * p / q) - sgn * path * dbb;
    const S sdn = (dn < S(0)) ? S(-1) : S(1);
    const S de1_ddn = -sgn * bb * dpath_dcos * sdn;
    mq = dq_de1 * de1_dq;
    mc = dq_de1 * de1_ddn;
}

// Alignment derivative of one record (6 values: dt, then w), see the header.
// g: dL/db_k^+, down: a_k - g_k (the part that comes from later records).
// Returns false for surfaces without an alignment model here (cylinders,
// lines).
template <typename S, bool W>
DPROP_HD bool alignment_contribution(const detector_view<S, W>& det,
                                     const dev_surface& sf, const S* b,
                                     vec3<S> dtds, S qop_in, S mc, const S* g,
                                     const S* down, S out[6]) {
    if (sf.shape != e_rectangle && sf.shape != e_trapezoid &&
        sf.shape != e_ring) {
        return false;
    }
    const dev_transform<S>& trf = det.transforms[sf.transform];
    const S cph = cos(b[2]), sph = sin(b[2]);
    const S cth = cos(b[3]), sth = sin(b[3]);
    const vec3<S> d{cph * sth, sph * sth, cth};
    const vec3<S> x = bound_to_free_pos(det, sf, b[0], b[1], d);
    const vec3<S> u = trf.x(), v = trf.y(), n = trf.z();
    const vec3<S> r = x - trf.translation();
    const S inv_nd = S(1) / dot(n, d);
    const vec3<S> nxr = cross(n, r);
    const vec3<S> uxr = cross(u, r);
    const vec3<S> vxr = cross(v, r);
    const vec3<S> nxd = cross(n, d);
    const S ud = dot(u, d), vd = dot(v, d);
    // ds / d(delta)
    const S s[6] = {n.x * inv_nd,    n.y * inv_nd,    n.z * inv_nd,
                    -nxr.x * inv_nd, -nxr.y * inv_nd, -nxr.z * inv_nd};
    const S ua[3] = {u.x, u.y, u.z}, va[3] = {v.x, v.y, v.z};
    const S uxra[3] = {uxr.x, uxr.y, uxr.z}, vxra[3] = {vxr.x, vxr.y, vxr.z};
    const S nxda[3] = {nxd.x, nxd.y, nxd.z};
    // local cartesian derivatives
    S lu[6], lv[6];
    for (int j = 0; j < 6; ++j) {
        lu[j] = ud * s[j] + ((j < 3) ? -ua[j] : uxra[j - 3]);
        lv[j] = vd * s[j] + ((j < 3) ? -va[j] : vxra[j - 3]);
    }
    S dl0[6], dl1[6];
    if (sf.shape == e_ring) {
        const S x0 = dot(u, r), x1 = dot(v, r);
        const S rho2 = x0 * x0 + x1 * x1;
        const S inv_rho = S(1) / sqrt(rho2);
        for (int j = 0; j < 6; ++j) {
            dl0[j] = (x0 * lu[j] + x1 * lv[j]) * inv_rho;
            dl1[j] = (x0 * lv[j] - x1 * lu[j]) / rho2;
        }
    } else {
        for (int j = 0; j < 6; ++j) {
            dl0[j] = lu[j];
            dl1[j] = lv[j];
        }
    }
    // incoming direction change per unit ds, in bound angles
    const S pphi = (-sph * dtds.x + cph * dtds.y) / sth;
    const S pth = cph * cth * dtds.x + sph * cth * dtds.y - sth * dtds.z;
    const S dn_s = dot(dtds, n);
    const S ratio = (qop_in != S(0)) ? S(1) - b[4] / qop_in : S(0);
    for (int j = 0; j < 6; ++j) {
        const S dphi = pphi * s[j];
        const S dth = pth * s[j];
        const S ddn = dn_s * s[j] + ((j < 3) ? S(0) : nxda[j - 3]);
        const S dq = mc * ddn;
        out[j] = g[0] * dl0[j] + g[1] * dl1[j] + g[2] * dphi + g[3] * dth +
                 g[4] * dq + (down[2] * dphi + down[3] * dth) * ratio +
                 down[4] * dq;
    }
    return true;
}

// Reverse sweep of one track.  Records are slot-major ([slot][n]); rec_bound
// and grad_bound are 6 component arrays (grad_bound entries may be null:
// zero gradient).  grad_free receives dL/d(x, y, z, t, tx, ty, tz, q/p);
// the direction part is tangent to the unit sphere at dir0 (the propagation
// treats the input direction as a unit vector).  Align(sf_index, out[6])
// receives the alignment contributions.
template <typename S, bool W, typename R, typename Align>
DPROP_HD void backward_track(const detector_view<S, W>& det,
                             const tape_view<S>& tp, uint64_t t,
                             uint32_t n_records, const uint64_t* rec_barcode,
                             const uint8_t* rec_flags,
                             const R* const* rec_bound,
                             const R* const* grad_bound, vec3<S> dir0,
                             S grad_free[8], Align&& align) {
    const uint64_t n = tp.n;
    const uint32_t count = n_records < tp.capacity ? n_records : tp.capacity;
    uint32_t first = count;
    for (uint32_t k = 0; k < count; ++k) {
        if (rec_flags[static_cast<uint64_t>(k) * n + t] & 1u) {
            first = k;
            break;
        }
    }
    for (int i = 0; i < 8; ++i) {
        grad_free[i] = S(0);
    }
    if (first == count) {
        return;
    }
    S a[6] = {S(0), S(0), S(0), S(0), S(0), S(0)};
    S c[6];
    for (uint32_t k = count; k-- > first;) {
        const uint64_t o = static_cast<uint64_t>(k) * n + t;
        if (!(rec_flags[o] & 1u)) {
            continue;
        }
        S g[6], b[6], down[6];
        for (int i = 0; i < 6; ++i) {
            g[i] = grad_bound[i] ? static_cast<S>(grad_bound[i][o]) : S(0);
            b[i] = static_cast<S>(rec_bound[i][o]);
            down[i] = a[i];
            a[i] = g[i] + down[i];
        }
        const bool repeat = tp.r(e_tape_repeat, k, t) != S(0);
        const S mq = tp.r(e_tape_mq, k, t);
        const S mc = tp.r(e_tape_mc, k, t);
        const uint64_t bc = rec_barcode[o];
        const uint32_t sfi = static_cast<uint32_t>((bc >> 27) & 0x1FFFFFu);
        const bool sf_ok =
            sfi < det.n_surfaces && det.surfaces[sfi].barcode == bc;
        if (sf_ok) {
            const dev_surface sf = det.surfaces[sfi];
            if (!repeat) {
                const vec3<S> dtds{tp.r(e_tape_dtds, k, t),
                                   tp.r(e_tape_dtds + 1, k, t),
                                   tp.r(e_tape_dtds + 2, k, t)};
                S contrib[6];
                if (alignment_contribution(det, sf, b, dtds,
                                           tp.r(e_tape_qop_in, k, t), mc, g,
                                           down, contrib)) {
                    align(sfi, contrib);
                }
            }
            // c = M^T a (the kick's q/p row through the incidence d.n)
            S m_loc0 = S(0), m_phi = S(0), m_th = S(0);
            if (mc != S(0)) {
                const S cph = cos(b[2]), sph = sin(b[2]);
                const S cth = cos(b[3]), sth = sin(b[3]);
                const vec3<S> n = surface_normal_at_bound(det, sf, b[0]);
                m_phi = mc * (-sth * sph * n.x + sth * cph * n.y);
                m_th = mc * (cth * cph * n.x + cth * sph * n.y - sth * n.z);
                if (sf.shape == e_concentric_cylinder) {
                    m_loc0 = mc * (-sin(b[0]) * cph * sth +
                                   cos(b[0]) * sph * sth);
                }
            }
            c[0] = a[0] + m_loc0 * a[4];
            c[2] = a[2] + m_phi * a[4];
            c[3] = a[3] + m_th * a[4];
        } else {
            c[0] = a[0];
            c[2] = a[2];
            c[3] = a[3];
        }
        c[1] = a[1];
        c[4] = mq * a[4];
        c[5] = a[5];
        if (k == first) {
            break;
        }
        // a = J_k^T c
        if (repeat) {
            for (int i = 0; i < 6; ++i) {
                a[i] = c[i];
            }
        } else {
            for (int j = 0; j < 5; ++j) {
                S acc = (j == 4) ? c[4] : S(0);
                for (int i = 0; i < 4; ++i) {
                    acc += tp.r(e_tape_g + i * 5 + j, k, t) * c[i];
                }
                a[j] = acc;
            }
            a[5] = c[5];
        }
    }
    // dL/dx0 = K^T c
    S gk[7];
    for (int j = 0; j < 7; ++j) {
        S acc = S(0);
        for (int i = 0; i < 5; ++i) {
            acc += tp.i(i * 7 + j, t) * c[i];
        }
        gk[j] = acc;
    }
    // project the direction gradient onto the tangent plane of dir0
    const S inv_len = S(1) / sqrt(dot(dir0, dir0));
    const vec3<S> u0 = dir0 * inv_len;
    const S radial = gk[3] * u0.x + gk[4] * u0.y + gk[5] * u0.z;
    grad_free[0] = gk[0];
    grad_free[1] = gk[1];
    grad_free[2] = gk[2];
    grad_free[3] = c[5];
    grad_free[4] = gk[3] - radial * u0.x;
    grad_free[5] = gk[4] - radial * u0.y;
    grad_free[6] = gk[5] - radial * u0.z;
    grad_free[7] = gk[6];
}

}  // namespace dprop
