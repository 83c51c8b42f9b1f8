/*
 * REFERENCE GPU BASELINE — measurement infrastructure only.  Types shared by
 * the kernel translation unit (ref_gpu.cu, nvcc) and the host driver
 * (ref_gpu_host.cpp, g++): the propagator type of the reference's CUDA
 * benchmark (tests/benchmarks/include/detray/benchmarks/device/cuda/
 * propagation_benchmark.hpp:50-72) over the toy detector.
 */
#pragma once

#include <cassert>

#include "detray/core/detector.hpp"
#include "detray/definitions/algebra.hpp"
#include "detray/detectors/toy_metadata.hpp"
#include "detray/navigation/caching_navigator.hpp"
#include "detray/propagator/actor_chain.hpp"
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

/// Enqueue one launch of the reference kernel on the legacy default stream.
int launch(const propagation::config& cfg,
           const typename toy_det_t::view_type& det_view,
           const const_field& field,
           const typename chain_t::state_tuple* states,
           vecmem::data::vector_view<track_t> tracks_view, uint8_t* status,
           unsigned int n);

}  // namespace refgpu
