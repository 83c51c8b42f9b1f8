/*
 * REFERENCE GPU BASELINE — measurement infrastructure only.  Types shared by
 * the kernel translation unit (ref_gpu.cu, nvcc) and the host driver
 * (ref_gpu_host.cpp, g++): the propagator type of the reference's CUDA
 * benchmark (tests/benchmarks/include/detray/benchmarks/device/cuda/
 * propagation_benchmark.hpp:50-72) over the toy detector, and the one of its
 * device propagation tutorial (tutorials/src/device/cuda/propagation.hpp,
 * propagation_kernel.cu:17-53: path-limit aborter, parameter updater with
 * the material interactor) in a field map.
 */
#pragma once

#include <cassert>

#include "detray/core/detector.hpp"
#include "detray/definitions/algebra.hpp"
#include "detray/detectors/toy_metadata.hpp"
#include "detray/navigation/caching_navigator.hpp"
#include "detray/propagator/actor_chain.hpp"
#include "detray/propagator/actors/aborters.hpp"
#include "detray/propagator/actors/parameter_updater.hpp"
#include "detray/propagator/actors/pointwise_material_interactor.hpp"
#include "detray/propagator/propagator.hpp"
#include "detray/propagator/rk_stepper.hpp"
#include "detray/tracks/tracks.hpp"

#include <cstdint>

namespace refgpu {

using namespace detray;

using scalar = float;
using algebra_t = detray::array<scalar>;
using toy_det_t = detector<toy_metadata<algebra_t>>;
using toy_dev_det_t = detector<toy_metadata<algebra_t>, device_container_types>;

// covfie::field_view<const backend> stand-in: at() returns the field vector
struct const_field {
    scalar b[3];
    DETRAY_HOST_DEVICE darray<scalar, 3> at(scalar, scalar, scalar) const {
        return {b[0], b[1], b[2]};
    }
};

using stepper_t =
    rk_stepper<const_field, algebra_t, unconstrained_step<scalar>,
               stepper_rk_policy<scalar>, stepping::void_inspector,
               static_cast<std::uint32_t>(
                   rk_stepper_flags::e_allow_covariance_transport)>;
using chain_t = actor_chain<actor::parameter_updater<
    algebra_t, actor::pointwise_material_interactor<algebra_t>>>;
using dev_propagator_t =
    propagator<stepper_t, caching_navigator<toy_dev_det_t>, chain_t>;
using track_t = free_track_parameters<algebra_t>;

// covfie field-view stand-in for the inhomogeneous configuration: a map on a
// regular (r, phi, z) node grid of float4 (B_r, B_phi, B_z, 0) in device
// memory, node index (iz * n_phi + iphi) * n_r + ir, trilinear in (r, phi,
// z) with clamping at the edges of r and z and a periodic phi axis; at()
// returns the Cartesian field.  The same definition as the oracle's field
// class (ref_field.hpp), evaluated in float as covfie's float maps are.
struct map_field {
    const float4* nodes;
    unsigned int n[3];
    scalar lo[3];
    scalar step_inv[3];  // r and z: (n - 1) / (hi - lo); phi: n / 2 pi

    DETRAY_HOST_DEVICE static void locate(scalar x, scalar l, scalar inv,
                                          unsigned int nn, unsigned int& i0,
                                          scalar& f) {
        if (nn < 2u) {
            i0 = 0u;
            f = 0.f;
            return;
        }
        const scalar umax = static_cast<scalar>(nn - 1u);
        scalar u = (x - l) * inv;
        u = u < 0.f ? 0.f : (u > umax ? umax : u);
        scalar fl = floorf(u);
        fl = fl > umax - 1.f ? umax - 1.f : fl;
        i0 = static_cast<unsigned int>(fl);
        f = u - fl;
    }

    DETRAY_HOST_DEVICE darray<scalar, 3> at(scalar x, scalar y,
                                             scalar z) const {
        const scalar r = sqrtf(x * x + y * y);
        unsigned int ir, iz, ip0 = 0u, ip1 = 0u;
        scalar fr, fz, fp = 0.f;
        locate(r, lo[0], step_inv[0], n[0], ir, fr);
        locate(z, lo[2], step_inv[2], n[2], iz, fz);
        if (n[1] > 1u) {
            const scalar np = static_cast<scalar>(n[1]);
            scalar u = (atan2f(y, x) - lo[1]) * step_inv[1];
            u = u - floorf(u / np) * np;
            const scalar fl = floorf(u);
            ip0 = static_cast<unsigned int>(fl) % n[1];
            ip1 = (ip0 + 1u) % n[1];
            fp = u - fl;
        }
        const unsigned int ir1 = n[0] > 1u ? ir + 1u : ir;
        const unsigned int iz1 = n[2] > 1u ? iz + 1u : iz;
        auto node = [&](unsigned int a, unsigned int p, unsigned int c) {
            return nodes[(static_cast<unsigned long long>(c) * n[1] + p) * n[0] + a];
        };
        const float4 c000 = node(ir, ip0, iz), c100 = node(ir1, ip0, iz);
        const float4 c010 = node(ir, ip1, iz), c110 = node(ir1, ip1, iz);
        const float4 c001 = node(ir, ip0, iz1), c101 = node(ir1, ip0, iz1);
        const float4 c011 = node(ir, ip1, iz1), c111 = node(ir1, ip1, iz1);
        scalar b[3];
        const float4* q[8] = {&c000, &c100, &c010, &c110,
                              &c001, &c101, &c011, &c111};
        for (int k = 0; k < 3; ++k) {
            auto g = [&](int i) {
                return k == 0 ? q[i]->x : (k == 1 ? q[i]->y : q[i]->z);
            };
            const scalar c00 = g(0) + fr * (g(1) - g(0));
            const scalar c10 = g(2) + fr * (g(3) - g(2));
            const scalar c01 = g(4) + fr * (g(5) - g(4));
            const scalar c11 = g(6) + fr * (g(7) - g(6));
            const scalar c0 = c00 + fp * (c10 - c00);
            const scalar c1 = c01 + fp * (c11 - c01);
            b[k] = c0 + fz * (c1 - c0);
        }
        const scalar cp = r > 0.f ? x / r : 1.f;
        const scalar sp = r > 0.f ? y / r : 0.f;
        return {b[0] * cp - b[1] * sp, b[0] * sp + b[1] * cp, b[2]};
    }
};

using map_stepper_t =
    rk_stepper<map_field, algebra_t, unconstrained_step<scalar>,
               stepper_rk_policy<scalar>, stepping::void_inspector,
               static_cast<std::uint32_t>(
                   rk_stepper_flags::e_allow_covariance_transport)>;
using limit_chain_t = actor_chain<
    actor::pathlimit_aborter<scalar>,
    actor::parameter_updater<algebra_t,
                             actor::pointwise_material_interactor<algebra_t>>>;
using map_propagator_t =
    propagator<map_stepper_t, caching_navigator<toy_dev_det_t>, limit_chain_t>;

/// Enqueue one launch of the tutorial-chain kernel in the field map on the
/// legacy default stream.
int launch_map(const propagation::config& cfg, scalar path_limit,
               const typename toy_det_t::view_type& det_view,
               const map_field& field,
               vecmem::data::vector_view<track_t> tracks_view,
               uint8_t* status, unsigned int n);

/// Enqueue one launch of the reference kernel on the legacy default stream.
int launch(const propagation::config& cfg,
           const typename toy_det_t::view_type& det_view,
           const const_field& field,
           const typename chain_t::state_tuple* states,
           vecmem::data::vector_view<track_t> tracks_view, uint8_t* status,
           unsigned int n);

}  // namespace refgpu
