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
//   energy loss in volume material        rk_stepper.hpp:146-231 (dqopds,
//                                          d2qopdsdqop), 536-567, 593-629,
//                                          760-800 (dqop_n/dqop1, dqopqop)
// Kernels for detectors without volume material are compiled without the
// energy-loss terms (VM = false): there q/p_n = q/p and dqopqop = 1.
#pragma once

#include "field.cuh"
#include "material.cuh"

namespace dprop {

// Non-trivial blocks of the 8x8 free transport Jacobian (25 values):
//   A = d(pos)/d(dir0), B = d(dir)/d(dir0), c = d(pos)/d(qop0),
//   d = d(dir)/d(qop0), e = d(qop)/d(qop0); everything else is identity.
// With the field gradient (Grad = true, the reference's 43-entry Jacobian,
// codegen/transport_jacobian.hpp) also P = d(pos)/d(pos0) and
// Q = d(dir)/d(pos0), which the gradient of an inhomogeneous field makes
// differ from the identity and zero.  Kept out of the default form so that
// kernels without the gradient do not carry 18 more live values.
template <typename S>
struct transport_jac_blocks {
    mat33<S> A;
    mat33<S> B;
    vec3<S> c;
    vec3<S> d;
    S e;

    DPROP_HD void reset_blocks() {
        for (int i = 0; i < 9; ++i) {
            A.m[i] = S(0);
        }
        B = identity33<S>();
        c = {S(0), S(0), S(0)};
        d = {S(0), S(0), S(0)};
        e = S(1);
    }
};

template <typename S, bool Grad = false>
struct transport_jac : transport_jac_blocks<S> {
    static constexpr bool gradient = false;
    DPROP_HD void reset() { this->reset_blocks(); }
};

template <typename S>
struct transport_jac<S, true> : transport_jac_blocks<S> {
    static constexpr bool gradient = true;
    mat33<S> P;
    mat33<S> Q;
    DPROP_HD void reset() {
        this->reset_blocks();
        P = identity33<S>();
        for (int i = 0; i < 9; ++i) {
            Q.m[i] = S(0);
        }
    }
};

template <typename S>
struct step_cfg {
    S min_stepsize;
    S rk_error_tol;
    uint32_t max_rk_updates;
    bool do_covariance_transport;
    bool field_gradient;  // use_field_gradient: kernels with Grad = true
    // energy loss in volume material (stepping::config)
    bool use_mean_loss;       // q/p of each RK stage from the previous one
    bool use_eloss_gradient;  // d(q/p)/d(q/p0) of the energy loss in the
                              // transport Jacobian
    S mass;                   // particle hypothesis
    bool electron;            // e+-: bremsstrahlung in the stopping power
};

// Per-track stepper state (rk_stepper::state + base_stepper::state); Grad:
// the transport Jacobian includes the field gradient.
template <typename S, bool Grad = false>
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
    transport_jac<S, Grad> jac;
    uint32_t n_trials;
    uint32_t n_steps;
};

template <typename S>
DPROP_HD S step_size_scaling(S tol, S err) {
    return min_(max_(sqrt(sqrt(tol / err)), S(0.25)), S(4));
}

// dt/ds of the state when no step was taken yet (rk_stepper::state::dtds)
template <typename S, bool Grad>
DPROP_HD vec3<S> current_dtds(const step_state<S, Grad>& st,
                              const field_view<S>& field) {
    if (st.path_length == 0.) {
        const vec3<S> b = field_at(field, st.pos);
        return st.qop * cross(st.dir, b);
    }
    return st.dtds;
}

// Central-difference gradient of the field, dB/dr (column i = dB/dr_i),
// with the reference's offset of 0.1 mm as a float literal
// (rk_stepper::evaluate_field_gradient, rk_stepper.hpp:958-997).
template <typename S>
DPROP_HD mat33<S> field_gradient(const field_view<S>& field, vec3<S> p) {
    const S delta = static_cast<S>(0.1f) * S(unit::mm);
    const S inv = S(1) / (S(2) * delta);
    mat33<S> g;
    for (int i = 0; i < 3; ++i) {
        const vec3<S> e{i == 0 ? delta : S(0), i == 1 ? delta : S(0),
                        i == 2 ? delta : S(0)};
        const vec3<S> b1 = field_at(field, p + e);
        const vec3<S> b2 = field_at(field, p - e);
        const vec3<S> d = (b1 - b2) * inv;
        g(0, i) = d.x;
        g(1, i) = d.y;
        g(2, i) = d.z;
    }
    return g;
}

template <typename S>
DPROP_HD mat33<S> matmul33(const mat33<S>& a, const mat33<S>& b) {
    mat33<S> r;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            S v = S(0);
            for (int k = 0; k < 3; ++k) {
                v += a(i, k) * b(k, j);
            }
            r(i, j) = v;
        }
    }
    return r;
}

// d(k_n)/d(r_1) of the four RKN stages with the field gradient (the
// reference's with-gradient transport, rk_stepper.hpp:872-938): k_n =
// qop (t_n x B(r_n)), so dk_n/dr_1 = qop (dt_n/dr_1 x B_n) - qop (dB_n/dr_n
// dr_n/dr_1 (x) t_n) with the stage tables dt_n/dr_1 and dr_n/dr_1; returns
// dF/dr = I + h^2/6 (dk1 + dk2 + dk3) and dG/dr = h/6 (dk1 + 2 (dk2 + dk3)
// + dk4).
template <typename S>
DPROP_HD void rk_position_derivatives(const field_view<S>& field, vec3<S> pos,
                                      vec3<S> pos1, vec3<S> pos2, S h,
                                      const S (&qn)[4], vec3<S> t0,
                                      vec3<S> t1, vec3<S> t2, vec3<S> t3,
                                      vec3<S> b_middle, vec3<S> b_last,
                                      mat33<S>& dFdr, mat33<S>& dGdr) {
    const S half_h = h * S(0.5);
    const S h2 = h * h;
    const mat33<S> I = identity33<S>();
    const mat33<S> g_ini = field_gradient(field, pos);
    const mat33<S> g_mid = field_gradient(field, pos1);
    const mat33<S> g_fin = field_gradient(field, pos2);
    mat33<S> k1 = colwise_cross(g_ini, t0);
    for (int i = 0; i < 9; ++i) {
        k1.m[i] *= -qn[0];
    }
    // dr_2/dr_1 = dr_3/dr_1 = I + h^2/8 dk1/dr1
    mat33<S> r23;
    for (int i = 0; i < 9; ++i) {
        r23.m[i] = I.m[i] + h2 * S(0.125) * k1.m[i];
    }
    const mat33<S> gr23 = matmul33(g_mid, r23);
    auto stage = [&](const mat33<S>& prev, S f, vec3<S> b, const mat33<S>& gr,
                     vec3<S> t, S qop) {
        mat33<S> a;
        for (int i = 0; i < 9; ++i) {
            a.m[i] = f * prev.m[i];
        }
        const mat33<S> x = colwise_cross(a, b);
        const mat33<S> y = colwise_cross(gr, t);
        mat33<S> r;
        for (int i = 0; i < 9; ++i) {
            r.m[i] = qop * x.m[i] - qop * y.m[i];
        }
        return r;
    };
    const mat33<S> k2 = stage(k1, half_h, b_middle, gr23, t1, qn[1]);
    const mat33<S> k3 = stage(k2, half_h, b_middle, gr23, t2, qn[2]);
    mat33<S> r4;
    for (int i = 0; i < 9; ++i) {
        r4.m[i] = I.m[i] + h2 * S(0.5) * k3.m[i];
    }
    const mat33<S> k4 = stage(k3, h, b_last, matmul33(g_fin, r4), t3, qn[3]);
    const S h_6 = h * static_cast<S>(1. / 6.);
    for (int i = 0; i < 9; ++i) {
        dFdr.m[i] = I.m[i] + h * h_6 * (k1.m[i] + k2.m[i] + k3.m[i]);
        dGdr.m[i] = h_6 * (k1.m[i] + S(2) * (k2.m[i] + k3.m[i]) + k4.m[i]);
    }
}

// One adaptive RKN4 step towards a surface at (signed) distance dist.  VM:
// the detector may carry volume material; vm is the material of the volume
// the track is in (NULL: none) and q the particle charge.
template <typename S, bool Grad, bool VM = false>
DPROP_HD bool rk_step(step_state<S, Grad>& st, S dist, const step_cfg<S>& cfg,
                      bool do_reset, const field_view<S>& field,
                      const dev_slab<S>* vm = nullptr, S q = S(1)) {
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
    // energy loss in the volume's material: q/p and d(q/p)/ds of each stage
    // (evaluate_dqopds); without material every stage has the start q/p
    const bool mat = VM && vm != nullptr;
    S qn[4] = {qop, qop, qop, qop};
    S dq[4] = {S(0), S(0), S(0), S(0)};
    auto stage_qop = [&](int i, S hs) {
        if constexpr (VM) {
            if (mat) {
                qn[i] = cfg.use_mean_loss ? qop + hs * dq[i - 1] : qop;
                dq[i] = eloss_dqopds(*vm, qn[i], q, cfg.mass, cfg.electron);
            }
        }
    };
    if constexpr (VM) {
        if (mat) {
            dq[0] = eloss_dqopds(*vm, qop, q, cfg.mass, cfg.electron);
        }
    }

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
        stage_qop(1, half_h);
        t1 = (h == S(0)) ? dir : dir + half_h * k0;
        k1 = qn[1] * cross(t1, b_middle);
        stage_qop(2, half_h);
        t2 = (h == S(0)) ? dir : dir + half_h * k1;
        k2 = qn[2] * cross(t2, b_middle);
        // last stage
        const vec3<S> pos2 = pos + h * t0 + (h2 * S(0.5)) * k2;
        b_last = field_at(field, pos2);
        stage_qop(3, h);
        t3 = (h == S(0)) ? dir : dir + h * k2;
        k3 = qn[3] * cross(t3, b_last);
        const S one_sixth = static_cast<S>(1. / 6.);
        const vec3<S> err_vec = (one_sixth * h2) * (k0 - k1 - k2 + k3);
        error = max_(norm(err_vec), S(1e-20));
        if (error <= four_tol) {
            break;
        }
        st.step_size = st.step_size * step_size_scaling(cfg.rk_error_tol, error);
    }
    st.dtds = k3;
    st.dqopds = dq[3];

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
    if constexpr (VM) {
        if (mat) {
            st.qop = qop + h_6 * (dq[0] + S(2) * (dq[1] + dq[2]) + dq[3]);
        }
    }
    st.path_length += static_cast<double>(h);
    st.abs_path_length += static_cast<double>(fabs(h));
    ++st.n_steps;

    if (cfg.do_covariance_transport) {
        const S half_h = h * S(0.5);
        // dqop_n/dqop1 and the energy loss's d(q/p)/d(q/p1) over the step
        // (both 1 without material or without the energy-loss gradient)
        S n1 = S(1), n2 = S(1), n3 = S(1);
        S dqopqop = S(1);
        if constexpr (VM) {
            if (mat && cfg.use_eloss_gradient) {
                const S g1 = eloss_d2qopdsdqop(*vm, qn[0], q, cfg.mass,
                                               cfg.electron);
                n1 = S(1) + half_h * g1;
                const S g2 = eloss_d2qopdsdqop(*vm, qn[1], q, cfg.mass,
                                               cfg.electron) *
                             n1;
                n2 = S(1) + half_h * g2;
                const S g3 = eloss_d2qopdsdqop(*vm, qn[2], q, cfg.mass,
                                               cfg.electron) *
                             n2;
                n3 = S(1) + h * g3;
                const S g4 = eloss_d2qopdsdqop(*vm, qn[3], q, cfg.mass,
                                               cfg.electron) *
                             n3;
                dqopqop = S(1) + h_6 * (g1 + S(2) * (g2 + g3) + g4);
            }
        }
        // dk_n/dqop
        const vec3<S> q0 = cross(t0, b_first);
        const vec3<S> q1 =
            n1 * cross(t1, b_middle) + (qn[1] * half_h) * cross(q0, b_middle);
        const vec3<S> q2 =
            n2 * cross(t2, b_middle) + (qn[2] * half_h) * cross(q1, b_middle);
        const vec3<S> q3 =
            n3 * cross(t3, b_last) + (qn[3] * h) * cross(q2, b_last);
        const vec3<S> dFdqop = (h * h_6) * (q0 + q1 + q2);
        const vec3<S> dGdqop = h_6 * (q0 + S(2) * (q1 + q2) + q3);

        // dk_n/dt
        const mat33<S> I = identity33<S>();
        mat33<S> d0 = colwise_cross(I, b_first);
        for (int k = 0; k < 9; ++k) {
            d0.m[k] *= qn[0];
        }
        mat33<S> tmp;
        for (int k = 0; k < 9; ++k) {
            tmp.m[k] = I.m[k] + half_h * d0.m[k];
        }
        mat33<S> d1 = colwise_cross(tmp, b_middle);
        for (int k = 0; k < 9; ++k) {
            d1.m[k] *= qn[1];
            tmp.m[k] = I.m[k] + half_h * d1.m[k];
        }
        mat33<S> d2 = colwise_cross(tmp, b_middle);
        for (int k = 0; k < 9; ++k) {
            d2.m[k] *= qn[2];
            tmp.m[k] = I.m[k] + h * d2.m[k];
        }
        mat33<S> d3 = colwise_cross(tmp, b_last);
        mat33<S> dFdt, dGdt;
        for (int k = 0; k < 9; ++k) {
            d3.m[k] *= qn[3];
            dFdt.m[k] = h * (I.m[k] + h_6 * (d0.m[k] + d1.m[k] + d2.m[k]));
            dGdt.m[k] = I.m[k] + h_6 * (d0.m[k] + S(2) * (d1.m[k] + d2.m[k]) +
                                        d3.m[k]);
        }

        // J <- D * J on the non-trivial blocks
        transport_jac<S, Grad>& J = st.jac;
        if constexpr (Grad) {
            // position columns: P' = dFdr P + dFdt Q, Q' = dGdr P + dGdt Q;
            // the direction and q/p columns take dFdr / dGdr below.  The
            // field gradients are taken where the reference takes them: it
            // advances the track before the Jacobian (rk_stepper.hpp:511-519)
            // and offsets the three points from the advanced position
            // (rk_stepper.hpp:885-897), so they lie one step further along
            // than the stages of the step
            const vec3<S> base = st.pos;
            const vec3<S> pos1 = base + half_h * t0 + (h * h * S(0.125)) * k0;
            const vec3<S> pos2 = base + h * t0 + (h * h * S(0.5)) * k2;
            mat33<S> dFdr, dGdr;
            rk_position_derivatives(field, base, pos1, pos2, h, qn, t0, t1,
                                    t2, t3, b_middle, b_last, dFdr, dGdr);
            mat33<S> nP, nQ;
            for (int r = 0; r < 3; ++r) {
                for (int c = 0; c < 3; ++c) {
                    S p = S(0), q = S(0);
                    for (int k = 0; k < 3; ++k) {
                        p += dFdr(r, k) * J.P(k, c) + dFdt(r, k) * J.Q(k, c);
                        q += dGdr(r, k) * J.P(k, c) + dGdt(r, k) * J.Q(k, c);
                    }
                    nP(r, c) = p;
                    nQ(r, c) = q;
                }
            }
            mat33<S> nA, nB;
            S ncv[3], ndv[3];
            const S jc[3] = {J.c.x, J.c.y, J.c.z};
            const S jd[3] = {J.d.x, J.d.y, J.d.z};
            const S fq[3] = {dFdqop.x, dFdqop.y, dFdqop.z};
            const S gq[3] = {dGdqop.x, dGdqop.y, dGdqop.z};
            for (int r = 0; r < 3; ++r) {
                for (int c = 0; c < 3; ++c) {
                    S a = S(0), b = S(0);
                    for (int k = 0; k < 3; ++k) {
                        a += dFdr(r, k) * J.A(k, c) + dFdt(r, k) * J.B(k, c);
                        b += dGdr(r, k) * J.A(k, c) + dGdt(r, k) * J.B(k, c);
                    }
                    nA(r, c) = a;
                    nB(r, c) = b;
                }
                S a = fq[r] * J.e, b = gq[r] * J.e;
                for (int k = 0; k < 3; ++k) {
                    a += dFdr(r, k) * jc[k] + dFdt(r, k) * jd[k];
                    b += dGdr(r, k) * jc[k] + dGdt(r, k) * jd[k];
                }
                ncv[r] = a;
                ndv[r] = b;
            }
            J.P = nP;
            J.Q = nQ;
            J.A = nA;
            J.B = nB;
            J.c = {ncv[0], ncv[1], ncv[2]};
            J.d = {ndv[0], ndv[1], ndv[2]};
            J.e = dqopqop * J.e;
        } else {
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
            J.e = dqopqop * J.e;
        }
    }
    return true;
}

}  // namespace dprop
