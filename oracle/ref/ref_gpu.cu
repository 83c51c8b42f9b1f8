/*
 * REFERENCE GPU BASELINE — measurement infrastructure only (see
 * ref_gpu_host.cpp).  The kernel body of the reference's
 * propagator_benchmark_kernel (tests/benchmarks/include/detray/benchmarks/
 * device/cuda/propagation_benchmark.cu:13-68, 256 threads per block,
 * __launch_bounds__(256, 4)), compiled for sm_100a from the reference's
 * headers; the one addition is a status byte per track (propagate()'s return
 * value) so that the work has an observable result.
 *
 * ref_map_kernel: the device propagation kernel of the reference's tutorial
 * (tutorials/src/device/cuda/propagation_kernel.cu:17-53): actor states
 * built per thread - path-limit aborter, parameter updater, material
 * interactor - over the same caching navigator and RK stepper in a field
 * map, one thread per track, 64 threads per block as the tutorial launches
 * it; the particle charge is set from each track as the benchmark kernel
 * does.
 */
#include <cuda_runtime.h>

#include "ref_gpu.hpp"

namespace refgpu {

__global__ void __launch_bounds__(256, 4)
    ref_propagation_kernel(const propagation::config cfg,
                           const typename toy_det_t::view_type det_view,
                           const const_field field,
                           const typename chain_t::state_tuple* states,
                           vecmem::data::vector_view<track_t> tracks_view,
                           uint8_t* status) {
    const toy_dev_det_t det(det_view);
    const vecmem::device_vector<track_t> tracks(tracks_view);
    const int gid = threadIdx.x + blockIdx.x * blockDim.x;
    if (gid >= static_cast<int>(tracks.size())) {
        return;
    }
    dev_propagator_t p{cfg};
    typename chain_t::state_tuple actor_states = *states;
    auto actor_state_refs = chain_t::setup_actor_states(actor_states);
    typename dev_propagator_t::state p_state(tracks.at(gid), field, det);
    auto& ptc = p_state.stepping().particle_hypothesis();
    p_state.set_particle(update_particle_hypothesis(ptc, tracks.at(gid)));
    status[gid] = p.propagate(p_state, actor_state_refs) ? 1u : 0u;
}

__global__ void ref_map_kernel(const propagation::config cfg,
                               const scalar path_limit,
                               const typename toy_det_t::view_type det_view,
                               const map_field field,
                               vecmem::data::vector_view<track_t> tracks_view,
                               uint8_t* status) {
    const int gid = threadIdx.x + blockIdx.x * blockDim.x;
    vecmem::device_vector<track_t> tracks(tracks_view);
    if (gid >= static_cast<int>(tracks.size())) {
        return;
    }
    const toy_dev_det_t det(det_view);
    map_propagator_t p{cfg};
    actor::pathlimit_aborter<scalar>::state aborter_state{path_limit};
    actor::parameter_updater_state<algebra_t> updater_state{cfg};
    actor::pointwise_material_interactor<algebra_t>::state interactor_state{};
    auto actor_states = detray::tie(aborter_state, updater_state,
                                    interactor_state);
    typename map_propagator_t::state state(tracks[gid], field, det);
    // the charge of each track's particle as the benchmark kernel sets it
    auto& ptc = state.stepping().particle_hypothesis();
    state.set_particle(update_particle_hypothesis(ptc, tracks[gid]));
    status[gid] = p.propagate(state, actor_states) ? 1u : 0u;
}

int launch_map(const propagation::config& cfg, scalar path_limit,
               const typename toy_det_t::view_type& det_view,
               const map_field& field,
               vecmem::data::vector_view<track_t> tracks_view,
               uint8_t* status, unsigned int n) {
    const unsigned int threads = 64u;
    const unsigned int blocks = (n + threads - 1u) / threads;
    ref_map_kernel<<<blocks, threads>>>(cfg, path_limit, det_view, field,
                                        tracks_view, status);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int launch(const propagation::config& cfg,
           const typename toy_det_t::view_type& det_view,
           const const_field& field,
           const typename chain_t::state_tuple* states,
           vecmem::data::vector_view<track_t> tracks_view, uint8_t* status,
           unsigned int n) {
    const unsigned int threads = 256u;
    const unsigned int blocks = (n + threads - 1u) / threads;
    ref_propagation_kernel<<<blocks, threads>>>(cfg, det_view, field, states,
                                                tracks_view, status);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace refgpu
