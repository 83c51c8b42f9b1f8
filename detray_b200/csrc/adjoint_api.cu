// Adjoint mode of the propagation and the reverse sweep: the C ABI entry
// points dprop_propagate_adjoint and dprop_backward (dprop.h).
//
// Kernels:
//   propagate_adjoint_kernel  the plain one-thread-per-track propagation that
//                             also writes the derivative tape of each track
//                             (core/adjoint.cuh: per transported record the
//                             4x5 surface-to-surface Jacobian block, the q/p
//                             kick derivatives, dt/ds and q/p before the
//                             kick; per track the start-to-first-surface
//                             Jacobian)
//   backward_kernel           one thread per track: the reverse sweep over
//                             its records (core/adjoint.cuh backward_track),
//                             alignment derivatives accumulated with fp64
//                             atomics per surface
#include <cuda_runtime.h>

#include <mutex>

#include "api_common.cuh"
#include "core/config.hpp"
#include "track_io.cuh"

using namespace dprop;
using dprop::api::fail;

namespace {

constexpr int k_adj_block = 128;

template <int MinBlocks, bool W, bool Grad>
__global__ void __launch_bounds__(k_adj_block, MinBlocks)
    propagate_adjoint_kernel(const __grid_constant__ detector_view<float, W> det,
                             const __grid_constant__ field_view<float> field,
                             const __grid_constant__ prop_cfg<float> cfg,
                             const __grid_constant__ api::io_ptrs<float> io,
                             const tape_view<float> tv, uint64_t n,
                             const uint32_t* __restrict__ order) {
    const uint64_t i =
        static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const uint64_t t = order ? static_cast<uint64_t>(order[i]) : i;
    api::run_one<float, true, float, W, Grad>(t, n, det, field, cfg, io, tv);
}

struct backward_io {
    const float* dir[3];
    const uint32_t* n_records;
    const uint64_t* rec_barcode;
    const uint8_t* rec_flags;
    const float* rec_bound[6];
    const float* grad_bound[6];
    float* grad_free[8];
    double* grad_align;
};

__global__ void __launch_bounds__(k_adj_block)
    backward_kernel(const detector_view<float> det, const tape_view<float> tv,
                    const backward_io io, uint64_t n) {
    const uint64_t t =
        static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) {
        return;
    }
    const vec3<float> dir0{io.dir[0][t], io.dir[1][t], io.dir[2][t]};
    float g[8];
    double* const ga = io.grad_align;
    backward_track(det, tv, t, io.n_records[t], io.rec_barcode, io.rec_flags,
                   io.rec_bound, io.grad_bound, dir0, g,
                   [ga](uint32_t sf, const float* v) {
                       if (ga != nullptr) {
                           double* dst = ga + 6u * static_cast<uint64_t>(sf);
                           for (int j = 0; j < 6; ++j) {
                               atomicAdd(dst + j, static_cast<double>(v[j]));
                           }
                       }
                   });
    for (int i = 0; i < 8; ++i) {
        if (io.grad_free[i]) {
            io.grad_free[i][t] = g[i];
        }
    }
}

// Library-owned, grow-only device scratch of the direction sort in adjoint
// mode (one per process; calls are serialised by the mutex on the host side
// and the scratch is only reused after the caller's stream reached it).
struct adj_sort_scratch {
    void* buf{nullptr};
    size_t bytes{0};
    int device{-1};
};
adj_sort_scratch g_adj_sort;
std::mutex g_adj_mutex;

template <int MB>
void launch_adjoint_mb(unsigned int grid, cudaStream_t st,
                       const dprop_detector* det,
                       const field_view<float>& field,
                       const prop_cfg<float>& cfg,
                       const api::io_ptrs<float>& io,
                       const tape_view<float>& tv, uint64_t n,
                       const uint32_t* order) {
    // with the field gradient: one register budget (8 CTAs per SM)
    if (cfg.step.field_gradient) {
        if (det->wires) {
            propagate_adjoint_kernel<8, true, true>
                <<<grid, k_adj_block, 0, st>>>(det->view_as<true>(), field,
                                               cfg, io, tv, n, order);
        } else {
            propagate_adjoint_kernel<8, false, true>
                <<<grid, k_adj_block, 0, st>>>(det->view_as<false>(), field,
                                               cfg, io, tv, n, order);
        }
        return;
    }
    if (det->wires) {
        propagate_adjoint_kernel<MB, true, false><<<grid, k_adj_block, 0, st>>>(
            det->view_as<true>(), field, cfg, io, tv, n, order);
    } else {
        propagate_adjoint_kernel<MB, false, false><<<grid, k_adj_block, 0, st>>>(
            det->view_as<false>(), field, cfg, io, tv, n, order);
    }
}

}  // namespace

extern "C" {

dprop_status dprop_propagate_adjoint(const dprop_config* cfg,
                                     const dprop_launch* lc,
                                     const dprop_detector* det,
                                     const dprop_field* field,
                                     const dprop_tracks* tracks,
                                     const dprop_results* results,
                                     const dprop_tape* tape, uint64_t n,
                                     void* stream) {
    if (!cfg || !det || !field || !tracks || !results || !tape) {
        return fail(DPROP_E_INVALID, "propagate_adjoint: NULL argument");
    }
    if (cfg->use_eloss_gradient || det->vol_material != nullptr) {
        return fail(DPROP_E_UNSUPPORTED,
                    "propagate_adjoint: the adjoint has no energy-loss term "
                    "for volume material (use_eloss_gradient, detectors with "
                    "volume material)");
    }
    if (cfg->max_iterations == 0u || cfg->max_records == 0u) {
        return fail(DPROP_E_INVALID,
                    "propagate_adjoint: max_iterations and max_records must "
                    "be > 0");
    }
    if (n == 0) {
        return DPROP_OK;
    }
    for (int i = 0; i < 3; ++i) {
        if (!tracks->pos[i] || !tracks->dir[i]) {
            return fail(DPROP_E_INVALID,
                        "propagate_adjoint: missing track array");
        }
    }
    if (!tracks->time || !tracks->qop || !results->status ||
        !results->n_records || !results->rec_barcode || !results->rec_flags) {
        return fail(DPROP_E_INVALID,
                    "propagate_adjoint: missing track/result array");
    }
    for (int i = 0; i < 6; ++i) {
        if (!results->rec_bound[i]) {
            return fail(DPROP_E_INVALID,
                        "propagate_adjoint: rec_bound arrays are required");
        }
    }
    if (!tape->rec || !tape->init) {
        return fail(DPROP_E_INVALID, "propagate_adjoint: missing tape array");
    }
    if (n > 0x7fffffffull * k_adj_block) {
        return fail(DPROP_E_INVALID, "propagate_adjoint: too many tracks");
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const api::io_ptrs<float> io = api::make_io<float>(*tracks, *results);
    tape_view<float> tv;
    tv.rec = static_cast<float*>(tape->rec);
    tv.init = static_cast<float*>(tape->init);
    tv.n = n;
    tv.capacity = cfg->max_records;

    std::lock_guard<std::mutex> lock(g_adj_mutex);
    const uint32_t* order = nullptr;
    if (lc && lc->sort_tracks) {
        const size_t need = api::sort_scratch_bytes(n);
        int dev = 0;
        DPROP_CUDA(cudaGetDevice(&dev));
        if (g_adj_sort.bytes < need || g_adj_sort.device != dev) {
            if (g_adj_sort.buf) {
                DPROP_CUDA(cudaStreamSynchronize(st));
                cudaFree(g_adj_sort.buf);
                g_adj_sort.buf = nullptr;
                g_adj_sort.bytes = 0;
            }
            DPROP_CUDA(cudaMalloc(&g_adj_sort.buf, need));
            g_adj_sort.bytes = need;
            g_adj_sort.device = dev;
        }
        const dprop_status s = api::enqueue_direction_sort(
            static_cast<const float*>(tracks->dir[0]),
            static_cast<const float*>(tracks->dir[1]),
            static_cast<const float*>(tracks->dir[2]),
            static_cast<const float*>(tracks->qop), n, g_adj_sort.buf,
            g_adj_sort.bytes, st, &order);
        if (s != DPROP_OK) {
            return s;
        }
    }
    const prop_cfg<float> pc = make_prop_cfg<float>(*cfg);
    const unsigned int grid =
        static_cast<unsigned int>((n + k_adj_block - 1) / k_adj_block);
    const int mb = api::occupancy_of(lc);
    if (mb == 8) {
        launch_adjoint_mb<8>(grid, st, det, field->view, pc, io, tv, n, order);
    } else if (mb == 12) {
        launch_adjoint_mb<12>(grid, st, det, field->view, pc, io, tv, n, order);
    } else {
        launch_adjoint_mb<16>(grid, st, det, field->view, pc, io, tv, n, order);
    }
    DPROP_CUDA(cudaGetLastError());
    return DPROP_OK;
}

dprop_status dprop_backward(const dprop_config* cfg, const dprop_detector* det,
                            const dprop_tracks* tracks,
                            const dprop_results* results,
                            const dprop_tape* tape,
                            const dprop_gradients* grads, uint64_t n,
                            void* stream) {
    if (!cfg || !det || !tracks || !results || !tape || !grads) {
        return fail(DPROP_E_INVALID, "backward: NULL argument");
    }
    if (cfg->max_records == 0u) {
        return fail(DPROP_E_INVALID, "backward: max_records must be > 0");
    }
    if (n == 0) {
        return DPROP_OK;
    }
    for (int i = 0; i < 3; ++i) {
        if (!tracks->dir[i]) {
            return fail(DPROP_E_INVALID, "backward: missing direction array");
        }
    }
    if (!results->n_records || !results->rec_barcode || !results->rec_flags) {
        return fail(DPROP_E_INVALID, "backward: missing result array");
    }
    for (int i = 0; i < 6; ++i) {
        if (!results->rec_bound[i]) {
            return fail(DPROP_E_INVALID, "backward: rec_bound arrays are required");
        }
    }
    if (!tape->rec || !tape->init) {
        return fail(DPROP_E_INVALID, "backward: missing tape array");
    }
    if (n > 0x7fffffffull * k_adj_block) {
        return fail(DPROP_E_INVALID, "backward: too many tracks");
    }
    backward_io io{};
    for (int i = 0; i < 3; ++i) {
        io.dir[i] = static_cast<const float*>(tracks->dir[i]);
    }
    io.n_records = results->n_records;
    io.rec_barcode = results->rec_barcode;
    io.rec_flags = results->rec_flags;
    for (int i = 0; i < 6; ++i) {
        io.rec_bound[i] = static_cast<const float*>(results->rec_bound[i]);
        io.grad_bound[i] = static_cast<const float*>(grads->grad_bound[i]);
    }
    for (int i = 0; i < 8; ++i) {
        io.grad_free[i] = static_cast<float*>(grads->grad_free[i]);
    }
    io.grad_align = grads->grad_align;
    tape_view<float> tv;
    tv.rec = static_cast<float*>(tape->rec);
    tv.init = static_cast<float*>(tape->init);
    tv.n = n;
    tv.capacity = cfg->max_records;
    const unsigned int grid =
        static_cast<unsigned int>((n + k_adj_block - 1) / k_adj_block);
    backward_kernel<<<grid, k_adj_block, 0, static_cast<cudaStream_t>(stream)>>>(
        det->view(), tv, io, n);
    DPROP_CUDA(cudaGetLastError());
    return DPROP_OK;
}

}  // extern "C"
