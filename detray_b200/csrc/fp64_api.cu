// fp64 propagation: the propagation core instantiated in double precision
// (the reference's full-fp64 build, DETRAY_CUSTOM_SCALARTYPE=double), for
// dprop_propagate with dprop_launch.precision = 8.  Track arrays, arithmetic
// and results are double; the field map nodes stay float4 (the reference's
// covfie field stores floats) and are interpolated in double.
//
// Kernels:
//   propagate_fp64_kernel<MB>  one thread per track, the whole propagation,
//                              register budget MB resident CTAs of 128
//                              threads per SM (8: 64 registers, 12: 40)
//   the round-based phase kernels of rounds_api.cu in double
//                              (dprop_launch.method = DPROP_METHOD_PERSISTENT)
#include <cuda_runtime.h>

#include <mutex>

#include "api_common.cuh"
#include "core/config.hpp"
#include "track_io.cuh"

using namespace dprop;
using dprop::api::fail;

namespace {

constexpr int k_f64_block = 128;

template <int MinBlocks, bool Grad = false>
__global__ void __launch_bounds__(k_f64_block, MinBlocks)
    propagate_fp64_kernel(const __grid_constant__ detector_view<double> det,
                          const __grid_constant__ field_view<double> field,
                          const __grid_constant__ prop_cfg<double> cfg,
                          const __grid_constant__ api::io_ptrs<double, double> io, uint64_t n,
                          const uint32_t* __restrict__ order) {
    const uint64_t i =
        static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const uint64_t t = order ? static_cast<uint64_t>(order[i]) : i;
    api::run_one<double, false, double, true, Grad>(t, n, det, field, cfg, io);
}

// library-owned grow-only sort scratch of fp64 launches
struct f64_sort_scratch {
    void* buf{nullptr};
    size_t bytes{0};
    int device{-1};
};
f64_sort_scratch g_f64_sort;
f64_sort_scratch g_f64_rounds;  // persistent method: slots and queues
std::mutex g_f64_mutex;

dprop_status ensure_f64(f64_sort_scratch& sc, size_t need,
                        cudaStream_t stream) {
    int dev = 0;
    DPROP_CUDA(cudaGetDevice(&dev));
    if (sc.bytes < need || sc.device != dev) {
        if (sc.buf) {
            DPROP_CUDA(cudaStreamSynchronize(stream));
            cudaFree(sc.buf);
            sc.buf = nullptr;
            sc.bytes = 0;
        }
        DPROP_CUDA(cudaMalloc(&sc.buf, need));
        sc.bytes = need;
        sc.device = dev;
    }
    return DPROP_OK;
}

}  // namespace

namespace dprop::api {

dprop_status propagate_fp64(const dprop_config& c, const dprop_launch* lc,
                            const dprop_detector* det, const dprop_field* field,
                            const dprop_tracks& tracks,
                            const dprop_results& results, uint64_t n,
                            cudaStream_t stream) {
    if (n > 0x7fffffffull * k_f64_block) {
        return fail(DPROP_E_INVALID, "propagate fp64: too many tracks");
    }
    const io_ptrs<double, double> io = make_io<double, double>(tracks, results);
    std::lock_guard<std::mutex> lock(g_f64_mutex);
    const uint32_t* order = nullptr;
    if (lc && lc->sort_tracks) {
        const dprop_status e =
            ensure_f64(g_f64_sort, sort_scratch_bytes(n), stream);
        if (e != DPROP_OK) {
            return e;
        }
        const dprop_status s = enqueue_direction_sort(
            io.trk[4], io.trk[5], io.trk[6], io.trk[7], n, g_f64_sort.buf,
            g_f64_sort.bytes, stream, &order);
        if (s != DPROP_OK) {
            return s;
        }
    }
    const prop_cfg<double> pc = make_prop_cfg<double>(c);
    if (lc && lc->method == DPROP_METHOD_PERSISTENT) {
        const size_t need = rounds_scratch_bytes_fp64(
            n, det->wires, staged_capacity(pc, io));
        const dprop_status e = ensure_f64(g_f64_rounds, need, stream);
        if (e != DPROP_OK) {
            return e;
        }
        return enqueue_rounds_fp64(lc, det, field, pc, io, n, order,
                                   g_f64_rounds.buf, g_f64_rounds.bytes,
                                   stream);
    }
    const unsigned int grid =
        static_cast<unsigned int>((n + k_f64_block - 1) / k_f64_block);
    if (c.use_field_gradient) {
        propagate_fp64_kernel<8, true><<<grid, k_f64_block, 0, stream>>>(
            det->view_d(), field->view_d, pc, io, n, order);
    } else if (occupancy_of(lc) >= 12) {
        propagate_fp64_kernel<12><<<grid, k_f64_block, 0, stream>>>(
            det->view_d(), field->view_d, pc, io, n, order);
    } else {
        propagate_fp64_kernel<8><<<grid, k_f64_block, 0, stream>>>(
            det->view_d(), field->view_d, pc, io, n, order);
    }
    DPROP_CUDA(cudaGetLastError());
    return DPROP_OK;
}

void release_fp64_scratch() {
    std::lock_guard<std::mutex> lock(g_f64_mutex);
    for (f64_sort_scratch* sc : {&g_f64_sort, &g_f64_rounds}) {
        cudaFree(sc->buf);
        *sc = f64_sort_scratch{};
    }
}

}  // namespace dprop::api
