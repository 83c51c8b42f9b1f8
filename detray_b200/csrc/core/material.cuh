// Energy loss in matter: the relativistic quantities of a track, the
// Bethe-Bloch stopping power and its derivative, the Landau width and the
// Highland / Rossi-Greisen scattering angle - used by the material
// interactor on surfaces and by the stepper in volumes with material.
//
// Reference: material/interaction.hpp:28-310,
// material/detail/relativistic_quantities.hpp; the stepper's energy loss
// rk_stepper::state::dqopds / d2qopdsdqop, propagator/rk_stepper.hpp:146-231.
#pragma once

#include "tables.cuh"

namespace dprop {

template <typename S>
struct rel_quantities {
    S qop, q2_over_beta2, beta2, beta_gamma, gamma, gamma2, E, Wmax;
};

template <typename S>
DPROP_HD rel_quantities<S> make_rq(S mass, S qop, S q) {
    rel_quantities<S> rq;
    rq.qop = qop;
    rq.q2_over_beta2 = q * q + (mass * qop) * (mass * qop);
    const S m_over_p = mass * ((q != S(0)) ? fabs(qop / q) : fabs(qop));
    const S p_over_m = S(1) / m_over_p;
    rq.beta2 = S(1) / (S(1) + m_over_p * m_over_p);
    rq.beta_gamma = p_over_m;
    rq.gamma = sqrt(S(1) + p_over_m * p_over_m);
    rq.gamma2 = rq.gamma * rq.gamma;
    rq.E = rq.gamma * mass;
    const S me = static_cast<S>(constant::m_e);
    const S mfrac = me / mass;
    rq.Wmax = (S(2) * me * rq.beta_gamma * rq.beta_gamma) /
              (S(1) + S(2) * rq.gamma * mfrac + mfrac * mfrac);
    return rq;
}

template <typename S>
DPROP_HD S eps_per_length(const dev_slab<S>& mat, const rel_quantities<S>& rq) {
    const S K = static_cast<S>(0.307075 * unit::MeV * unit::cm2);
    return S(0.5) * K * mat.molar_electron_density * rq.q2_over_beta2;
}

template <typename S>
DPROP_HD S delta_half(const dev_slab<S>& mat, const rel_quantities<S>& rq) {
    if (mat.has_density_effect == S(0)) {
        if (rq.beta_gamma < S(10)) {
            return S(0);
        }
        const S plasma = static_cast<S>(28.816 * unit::eV) *
                         sqrt(S(1000) * mat.molar_electron_density);
        return log(rq.beta_gamma * plasma / mat.mean_excitation_energy) -
               S(0.5);
    }
    const S x = log10(rq.beta_gamma);
    S delta = S(0);
    if (x >= mat.density_x0) {
        delta = S(2) * static_cast<S>(constant::ln10) * x - mat.density_c;
        if (x < mat.density_x1) {
            delta += mat.density_a * pow(mat.density_x1 - x, mat.density_m);
        }
    }
    return S(0.5) * delta;
}

template <typename S>
DPROP_HD S bethe_bloch(const dev_slab<S>& mat, const rel_quantities<S>& rq) {
    const S epl = eps_per_length(mat, rq);
    if (epl <= S(0)) {
        return S(0);
    }
    const S dhalf = delta_half(mat, rq);
    const S I = mat.mean_excitation_energy;
    const S u = S(2) * static_cast<S>(constant::m_e) * rq.beta_gamma *
                rq.beta_gamma;
    const S A = S(0.5) * log(u * rq.Wmax / (I * I));
    return S(2) * epl * (A - rq.beta2 - dhalf);
}

template <typename S>
DPROP_HD S landau_sigma_qop(S path_segment, const dev_slab<S>& mat,
                            const rel_quantities<S>& rq, S q) {
    const S fwhm = S(4) * eps_per_length(mat, rq) * path_segment;
    const S sigmaE = S(0.5) * static_cast<S>(constant::inv_sqrt2) * fwhm /
                     sqrt(static_cast<S>(constant::ln2));
    const S p_inv = rq.qop / q;
    return sqrt(rq.q2_over_beta2) * p_inv * p_inv * sigmaE;
}

template <typename S>
DPROP_HD S scattering_theta0(S x_over_x0, const rel_quantities<S>& rq, S q,
                             bool electron) {
    if (x_over_x0 <= S(0)) {
        return S(0);
    }
    const S mom_inv = fabs(rq.qop / q);
    const S t = sqrt(x_over_x0 * rq.q2_over_beta2);
    if (electron) {
        return static_cast<S>(17.5 * unit::MeV) * mom_inv * t *
               (S(1) + S(0.125) * log10(S(10) * x_over_x0));
    }
    return static_cast<S>(13.6 * unit::MeV) * mom_inv * t *
           (S(1) + S(0.038) * S(2) * log(t));
}

// d(-dE/dx)/d(q/p) of the mean Bethe-Bloch stopping power (the formula of
// interaction::derive_bethe_bloch, material/interaction.hpp:105-153).
// Without density-effect data the derivative of delta/2 is, with
// RefDelta = false, that of the forward formula (zero below beta*gamma =
// 10, -1/(q/p) above: the adjoint differentiates what the forward pass
// computes); with RefDelta = true it is the reference's -1/(q/p) at every
// beta*gamma (relativistic_quantities::derive_delta_half,
// material/detail/relativistic_quantities.hpp:193-229), which the stepper's
// energy-loss gradient uses.
template <typename S, bool RefDelta = false>
DPROP_HD S bethe_bloch_dqop(const dev_slab<S>& mat, const rel_quantities<S>& rq,
                            S bethe) {
    const S epl = eps_per_length(mat, rq);
    if (epl <= S(0)) {
        return S(0);
    }
    const S first = S(2) / (rq.qop * rq.gamma2) * bethe;
    const S dA = S(-1) / (S(2) * rq.qop) * (S(4) - rq.Wmax / rq.E);
    const S dB = S(-2) * rq.beta2 / (rq.qop * rq.gamma2);
    S dC;
    if (mat.has_density_effect == S(0)) {
        dC = (RefDelta || !(rq.beta_gamma < S(10))) ? S(-1) / rq.qop : S(0);
    } else {
        const S x = log10(rq.beta_gamma);
        S delta = S(0);
        if (x >= mat.density_x0) {
            delta = S(-2) / rq.qop;
            if (x < mat.density_x1) {
                delta += mat.density_a * mat.density_m /
                         (rq.qop * static_cast<S>(constant::ln10)) *
                         pow(mat.density_x1 - x, mat.density_m - S(1));
            }
        }
        dC = S(0.5) * delta;
    }
    return first + S(2) * epl * (dA - dB - dC);
}

// Total stopping power <-dE/dx> (interaction::compute_stopping_power,
// interaction.hpp:28-42): Bethe-Bloch, plus Rossi's bremsstrahlung
// approximation gamma m / X0 for electrons and positrons.
template <typename S>
DPROP_HD S stopping_power(const dev_slab<S>& mat, const rel_quantities<S>& rq,
                          S mass, bool electron) {
    S sp = bethe_bloch(mat, rq);
    if (electron) {
        sp += rq.gamma * mass / mat.X0;
    }
    return sp;
}

// d(q/p)/ds in a volume's material, (q/p)^3 E <-dE/dx> / q^2
// (rk_stepper::state::dqopds, rk_stepper.hpp:158-190).
template <typename S>
DPROP_HD S eloss_dqopds(const dev_slab<S>& mat, S qop, S q, S mass,
                        bool electron) {
    const S p = q / qop;
    const S E = sqrt(p * p + mass * mass);
    const rel_quantities<S> rq = make_rq(mass, qop, q);
    const S sp = stopping_power(mat, rq, mass, electron);
    return qop * qop * qop * E * sp / (q * q);
}

// d(d(q/p)/ds)/d(q/p) (rk_stepper::state::d2qopdsdqop, rk_stepper.hpp:
// 195-230, Eq. 3.12 of JINST 4 (2009) P04016): with g = dE/ds,
// dqopds * (1/qop (3 - p^2/E^2) + dg/dqop / g).
template <typename S>
DPROP_HD S eloss_d2qopdsdqop(const dev_slab<S>& mat, S qop, S q, S mass,
                             bool electron) {
    const S p = q / qop;
    const S p2 = p * p;
    const S E2 = p2 + mass * mass;
    const rel_quantities<S> rq = make_rq(mass, qop, q);
    const S bb = bethe_bloch(mat, rq);
    S sp = bb;
    S dsp = bethe_bloch_dqop<S, true>(mat, rq, bb);
    if (electron) {
        sp += rq.gamma * mass / mat.X0;
        dsp += -rq.beta2 * rq.gamma / rq.qop * mass / mat.X0;
    }
    const S g = -sp;
    const S dgdqop = -dsp;
    const S dqopds = qop * qop * qop * sqrt(E2) * sp / (q * q);
    return dqopds * (S(1) / qop * (S(3) - p2 / E2) + S(1) / g * dgdqop);
}

}  // namespace dprop
