// Runge-Kutta-Nystrom 4th order stepper with adaptive step-size control and
// transport-Jacobian update, one track per thread.
//
// Reference: rk_stepper::step and helpers
//   step / error control / step scaling   propagator/rk_stepper.hpp:273-530
//   evaluate_dtds / evaluate_dqopds        rk_stepper.hpp:533-590
//   advance_track                          rk_stepper.hpp:593-629
//   advance_jacobian                       rk_stepper.hpp:632-956
//   transport Jacobian structure           codegen/detray-sympy/detray_sympy/
//                                          matrices.py (D * J with the
//                                          identity sub-structure)
// Volume material (dqop/ds) is not on the device path: the supported
// detectors carry surface material only, so qop_n = qop and dqopqop = 1.
#pragma once

#include "field.cuh"

namespace dprop {

// Non-trivial blocks of the 8x8 free transport Jacobian (25 values):
//   A = d(pos)/d(dir0), B = d(dir)/d(dir0), c = d(pos)/d(qop0),
//   d = d(dir)/d(qop0), e = d(qop)/d(qop0); everything else is identity.
template <typename S>
struct transport_jac {
    mat33<S> A;
    mat33<S> B;
    vec3<S> c;
    vec3<S> d;
    S e;

    DPROP_HD void reset() {
        for (int i = 0; i < 9; ++i) {
            A.m[i] = S(0);
        }
        B = identity33<S>();
        c = {S(0), S(0), S(0)};
        d = {S(0), S(0), S(0)};
        e = S(1);
    }
};

template <typename S>
struct step_cfg {
    S min_stepsize;
    S rk_error_tol;
    uint32_t max_rk_updates;
    bool do_covariance_transport;
};

// Per-track stepper state (rk_stepper::state + base_stepper::state)
template <typename S>
struct step_state {
    vec3<S> pos;
    vec3<S> dir;
    S qop;
    S time;
    double path_length;      // accumulated in fp64 on the device
    double abs_path_length;
    S step_size;
    S next_step_size;
    vec3<S> dtds;            // dt/ds at the end of the last step
    S dqopds;
    S constraint;            // min over the step constraints (accuracy, aborter)
    transport_jac<S> jac;
    uint32_t n_trials;
    uint32_t n_steps;
};

template <typename S>
DPROP_HD S step_size_scaling(S tol, S err) {
    return min_(max_(sqrt(sqrt(tol / err)), S(0.25)), S(4));
}

// dt/ds of the state when no step was taken yet (rk_stepper::state::dtds)
template <typename S>
DPROP_HD vec3<S> current_dtds(const step_state<S>& st,
                              const field_view<S>& field) {
    if (st.path_length == 0.) {
        const vec3<S> b = field_at(field, st.pos);
        return st.qop * cross(st.dir, b);
    }
    return st.dtds;
}

// One adaptive RKN4 step towards a surface at (signed) distance dist.
template <typename S>
DPROP_HD bool rk_step(step_state<S>& st, S dist, const step_cfg<S>& cfg,
                      bool do_reset, const field_view<S>& field) {
    const S um = S(unit::um);
    if (fabs(dist) < um) {
        if (fabs(st.next_step_size) < cfg.min_stepsize) {
            st.next_step_size = copysign(cfg.min_stepsize, dist);
        }
        return true;
    }
    if (do_reset) {
        st.step_size = dist;
    } else if (st.next_step_size > S(0)) {
        st.step_size = min_(st.next_step_size, dist);
    } else {
        st.step_size = max_(st.next_step_size, dist);
    }
    const S min_step = min_(fabs(st.step_size), cfg.min_stepsize);
    const vec3<S> pos = st.pos;
    const vec3<S> dir = st.dir;
    const S qop = st.qop;

    // first stage
    const vec3<S> b_first = field_at(field, pos);
    const vec3<S> t0 = dir;
    const vec3<S> k0 = qop * cross(t0, b_first);

    vec3<S> b_middle{S(0), S(0), S(0)};
    vec3<S> b_last{S(0), S(0), S(0)};
    vec3<S> t1 = t0, t2 = t0, t3 = t0;
    vec3<S> k1 = k0, k2 = k0, k3 = k0;

    S error = S(1e20);
    const S four_tol = S(4) * cfg.rk_error_tol;
    for (uint32_t i = 0u; i < cfg.max_rk_updates; ++i) {
        ++st.n_trials;
        const S h = st.step_size;
        const S h2 = h * h;
        const S half_h = h * S(0.5);
        // second and third stage share the field at the mid point
        const vec3<S> pos1 = pos + half_h * t0 + (h2 * S(0.125)) * k0;
        b_middle = field_at(field, pos1);
        t1 = (h == S(0)) ? dir : dir + half_h * k0;
        k1 = qop * cross(t1, b_middle);
        t2 = (h == S(0)) ? dir : dir + half_h * k1;
        k2 = qop * cross(t2, b_middle);
        // last stage
        const vec3<S> pos2 = pos + h * t0 + (h2 * S(0.5)) * k2;
        b_last = field_at(field, pos2);
        t3 = (h == S(0)) ? dir : dir + h * k2;
        k3 = qop * cross(t3, b_last);
        const S one_sixth = static_cast<S>(1. / 6.);
        const vec3<S> err_vec = (one_sixth * h2) * (k0 - k1 - k2 + k3);
        error = max_(norm(err_vec), S(1e-20));
        if (error <= four_tol) {
            break;
        }
        st.step_size = st.step_size * step_size_scaling(cfg.rk_error_tol, error);
    }
    st.dtds = k3;
    st.dqopds = S(0);

    // step constraints (constrained_step::size, signed by the direction)
    const S dir_sign = st.step_size >= S(0) ? S(1) : S(-1);
    const S max_step = dir_sign * st.constraint;
    if (fabs(st.step_size) > fabs(max_step)) {
        st.step_size = max_step;
    }
    if (fabs(st.step_size) < min_step) {
        st.step_size = copysign(min_step, st.step_size);
    }
    st.next_step_size =
        st.step_size * step_size_scaling(cfg.rk_error_tol, error);
    if (fabs(st.next_step_size) < cfg.min_stepsize) {
        st.next_step_size = copysign(cfg.min_stepsize, st.next_step_size);
    }

    // advance the track (Eq. 82 of NIM 178 (1981) 203)
    const S h = st.step_size;
    const S h_6 = h * static_cast<S>(1. / 6.);
    st.pos = pos + h * (t0 + h_6 * (k0 + k1 + k2));
    st.dir = normalize(dir + h_6 * (k0 + S(2) * (k1 + k2) + k3));
    st.path_length += static_cast<double>(h);
    st.abs_path_length += static_cast<double>(fabs(h));
    ++st.n_steps;

    if (cfg.do_covariance_transport) {
        const S half_h = h * S(0.5);
        // dk_n/dqop (qop_n = qop, no energy-loss gradient)
        const vec3<S> q0 = cross(t0, b_first);
        const vec3<S> q1 = cross(t1, b_middle) + (qop * half_h) * cross(q0, b_middle);
        const vec3<S> q2 = cross(t2, b_middle) + (qop * half_h) * cross(q1, b_middle);
        const vec3<S> q3 = cross(t3, b_last) + (qop * h) * cross(q2, b_last);
        const vec3<S> dFdqop = (h * h_6) * (q0 + q1 + q2);
        const vec3<S> dGdqop = h_6 * (q0 + S(2) * (q1 + q2) + q3);

        // dk_n/dt
        const mat33<S> I = identity33<S>();
        mat33<S> d0 = colwise_cross(I, b_first);
        for (int k = 0; k < 9; ++k) {
            d0.m[k] *= qop;
        }
        mat33<S> tmp;
        for (int k = 0; k < 9; ++k) {
            tmp.m[k] = I.m[k] + half_h * d0.m[k];
        }
        mat33<S> d1 = colwise_cross(tmp, b_middle);
        for (int k = 0; k < 9; ++k) {
            d1.m[k] *= qop;
            tmp.m[k] = I.m[k] + half_h * d1.m[k];
        }
        mat33<S> d2 = colwise_cross(tmp, b_middle);
        for (int k = 0; k < 9; ++k) {
            d2.m[k] *= qop;
            tmp.m[k] = I.m[k] + h * d2.m[k];
        }
        mat33<S> d3 = colwise_cross(tmp, b_last);
        mat33<S> dFdt, dGdt;
        for (int k = 0; k < 9; ++k) {
            d3.m[k] *= qop;
            dFdt.m[k] = h * (I.m[k] + h_6 * (d0.m[k] + d1.m[k] + d2.m[k]));
            dGdt.m[k] = I.m[k] + h_6 * (d0.m[k] + S(2) * (d1.m[k] + d2.m[k]) +
                                        d3.m[k]);
        }

        // J <- D * J on the non-trivial blocks
        transport_jac<S>& J = st.jac;
        mat33<S> nA, nB;
        vec3<S> nc, nd;
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c) {
                S a = J.A(r, c);
                S b = S(0);
                for (int k = 0; k < 3; ++k) {
                    a += dFdt(r, k) * J.B(k, c);
                    b += dGdt(r, k) * J.B(k, c);
                }
                nA(r, c) = a;
                nB(r, c) = b;
            }
        }
        const S jd[3] = {J.d.x, J.d.y, J.d.z};
        const S fq[3] = {dFdqop.x, dFdqop.y, dFdqop.z};
        const S gq[3] = {dGdqop.x, dGdqop.y, dGdqop.z};
        const S jc[3] = {J.c.x, J.c.y, J.c.z};
        S ncv[3], ndv[3];
        for (int r = 0; r < 3; ++r) {
            S a = jc[r] + fq[r] * J.e;
            S b = gq[r] * J.e;
            for (int k = 0; k < 3; ++k) {
                a += dFdt(r, k) * jd[k];
                b += dGdt(r, k) * jd[k];
            }
            ncv[r] = a;
            ndv[r] = b;
        }
        nc = {ncv[0], ncv[1], ncv[2]};
        nd = {ndv[0], ndv[1], ndv[2]};
        J.A = nA;
        J.B = nB;
        J.c = nc;
        J.d = nd;
        // J.e unchanged: dqopqop = 1
    }
    return true;
}

}  // namespace dprop
