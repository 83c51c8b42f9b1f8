/*
 * REFERENCE GPU BASELINE — measurement infrastructure only (see
 * ref_gpu_host.cpp).  The kernel body of the reference's
 * propagator_benchmark_kernel (tests/benchmarks/include/detray/benchmarks/
 * device/cuda/propagation_benchmark.cu:13-68, 256 threads per block,
 * __launch_bounds__(256, 4)), compiled for sm_100a from the reference's
 * headers; the one addition is a status byte per track (propagate()'s return
 * value) so that the work has an observable result.
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
