// C ABI of the B200 track propagator (include/detray_b200/dprop.h) and the
// propagation kernels.
//
// Kernels:
//   propagate_plain_kernel       one thread per track, the whole propagation;
//                                the same launch form as the reference's
//                                propagator_benchmark_kernel
//                                (tests/benchmarks/include/detray/benchmarks/
//                                device/cuda/propagation_benchmark.cu:13-68)
// The persistent method's round-based phase kernels are in rounds_api.cu.
// Both write the slot-major records of dprop_results.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "api_common.cuh"
#include "core/config.hpp"
#include "core/convert.hpp"
#include "track_io.cuh"

using namespace dprop;
using dprop::api::io_ptrs;
using dprop::api::make_io;
using dprop::api::run_one;

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace dprop::api {

dprop_status fail(dprop_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

dprop_status cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return (e == cudaErrorMemoryAllocation) ? DPROP_E_OOM : DPROP_E_CUDA;
}

}  // namespace dprop::api

using dprop::api::cuda_fail;
using dprop::api::fail;

namespace {

template <typename T>
dprop_status upload(const std::vector<T>& h, T** d) {
    *d = nullptr;
    if (h.empty()) {
        return DPROP_OK;
    }
    DPROP_CUDA(cudaMalloc(reinterpret_cast<void**>(d), h.size() * sizeof(T)));
    DPROP_CUDA(cudaMemcpy(*d, h.data(), h.size() * sizeof(T),
                          cudaMemcpyHostToDevice));
    return DPROP_OK;
}

}  // namespace

namespace {

// Device scratch owned by the library for the host-buffer entry point:
// grow-only, reused across calls (not thread-safe across host threads).
struct host_path_scratch {
    void* buf{nullptr};
    size_t bytes{0};
    unsigned int* counter{nullptr};
};
host_path_scratch g_scratch;

dprop_status ensure_scratch(size_t bytes) {
    if (g_scratch.bytes >= bytes) {
        return DPROP_OK;
    }
    if (g_scratch.buf) {
        cudaFree(g_scratch.buf);
        g_scratch.buf = nullptr;
        g_scratch.bytes = 0;
    }
    DPROP_CUDA(cudaMalloc(&g_scratch.buf, bytes));
    g_scratch.bytes = bytes;
    return DPROP_OK;
}

// Library-owned device scratch of the direction sort and of the persistent
// method (grow-only).
struct sort_scratch {
    void* buf{nullptr};
    size_t bytes{0};
};
sort_scratch g_sort;
sort_scratch g_rounds;

// Sort key of a track, 20 bits: 7 bits of theta (major), 8 bits of phi, the
// charge sign and 4 bits of log10(pT / GeV) over [-1, 2].  Tracks that share
// a key cell start in the same direction with similar curvature, so the
// lanes of a warp cross the same modules at the same loop iterations.
template <typename In>
__global__ void direction_key_kernel(const In* __restrict__ dx,
                                     const In* __restrict__ dy,
                                     const In* __restrict__ dz,
                                     const In* __restrict__ dq, uint64_t n,
                                     uint32_t* __restrict__ keys,
                                     uint32_t* __restrict__ idx) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const float x = static_cast<float>(dx[i]);
    const float y = static_cast<float>(dy[i]);
    const float z = static_cast<float>(dz[i]);
    const float q = static_cast<float>(dq[i]);
    const float rho = sqrtf(x * x + y * y);
    const float theta = atan2f(rho, z);
    const float phi = atan2f(y, x);
    int tb = static_cast<int>(theta * (128.f / 3.14159265f));
    int pb = static_cast<int>((phi + 3.14159265f) * (256.f / 6.2831853f));
    tb = tb < 0 ? 0 : (tb > 127 ? 127 : tb);
    pb = pb < 0 ? 0 : (pb > 255 ? 255 : pb);
    // pT = rho / |q/p| (unit direction); non-finite or zero q/p -> top bin
    const float lpt = log10f(rho / fabsf(q));
    int kb = static_cast<int>((lpt + 1.f) * (16.f / 3.f));
    kb = !(lpt == lpt) ? 15 : (kb < 0 ? 0 : (kb > 15 ? 15 : kb));
    const uint32_t sign = (q < 0.f) ? 1u : 0u;
    keys[i] = (static_cast<uint32_t>(tb) << 13) |
              (static_cast<uint32_t>(pb) << 5) | (sign << 4) |
              static_cast<uint32_t>(kb);
    idx[i] = static_cast<uint32_t>(i);
}


// Threads per CTA and the minimum resident CTAs per SM the register
// allocation targets (__launch_bounds__); overridable at build time for
// tuning sweeps.
#ifndef DPROP_BLOCK
#define DPROP_BLOCK 128
#endif
#ifndef DPROP_MIN_BLOCKS
// 12 resident CTAs of 128 threads per SM (40 registers per thread): measured
// on B200 to hide the latency of the divergent navigation better than fewer
// warps with more registers, despite the extra spills to L1
#define DPROP_MIN_BLOCKS 12
#endif
constexpr int k_plain_block = DPROP_BLOCK;
// Largest CTA a plain launch may use (dprop_launch.block_size): the kernels
// are compiled for it, with the resident-CTA count scaled so that the
// register budget is the one of MinBlocks CTAs of k_plain_block threads.
constexpr int k_plain_max_block = 256;
static_assert(k_plain_max_block % k_plain_block == 0,
              "the largest plain CTA is a multiple of the default one");

// One instantiation per register budget: MinBlocks resident CTAs of 128
// threads per SM -> 8: 64 registers, 12: 40 registers, 16: 32 registers per
// thread (the rest spills to L1).  More resident warps hide more of the
// navigation's memory and instruction-fetch latency; the best budget depends
// on the workload (constant field vs field map), so it is a launch choice.
template <typename In, int MinBlocks = DPROP_MIN_BLOCKS, bool W = true,
          bool Grad = false>
__global__ void __launch_bounds__(
    k_plain_max_block, MinBlocks * k_plain_block / k_plain_max_block)
    propagate_plain_kernel(const __grid_constant__ detector_view<float, W> det,
                           const __grid_constant__ field_view<float> field,
                           const __grid_constant__ prop_cfg<float> cfg,
                           const __grid_constant__ io_ptrs<In> io,
                           uint64_t n, const uint32_t* __restrict__ order) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const uint64_t t = order ? static_cast<uint64_t>(order[i]) : i;
    run_one<In, false, float, W, Grad>(t, n, det, field, cfg, io);
}

}  // namespace

namespace dprop::api {

// register budget of a launch: resident CTAs per SM in {8, 12, 16}
int occupancy_of(const dprop_launch* lc) {
    const uint32_t v = (lc && lc->ctas_per_sm) ? lc->ctas_per_sm
                                               : static_cast<uint32_t>(DPROP_MIN_BLOCKS);
    return v <= 8u ? 8 : (v <= 12u ? 12 : 16);
}

size_t sort_scratch_bytes(uint64_t n) {
    size_t temp = 0;
    cub::DeviceRadixSort::SortPairs(
        nullptr, temp, static_cast<const uint32_t*>(nullptr),
        static_cast<uint32_t*>(nullptr), static_cast<const uint32_t*>(nullptr),
        static_cast<uint32_t*>(nullptr), static_cast<int>(n), 0, 20);
    const size_t arr = ((n * sizeof(uint32_t)) + 255) & ~size_t(255);
    return 4 * arr + temp + 256;
}

template <typename In>
dprop_status enqueue_sort(const In* dx, const In* dy, const In* dz,
                          const In* dq, uint64_t n, void* scratch, size_t scratch_bytes,
                          cudaStream_t stream, const uint32_t** order) {
    if (n > 0x7fffffffull) {
        return fail(DPROP_E_INVALID, "sort_tracks: too many tracks");
    }
    const size_t arr = ((n * sizeof(uint32_t)) + 255) & ~size_t(255);
    char* p = static_cast<char*>(scratch);
    uint32_t* keys_in = reinterpret_cast<uint32_t*>(p);
    uint32_t* keys_out = reinterpret_cast<uint32_t*>(p + arr);
    uint32_t* idx_in = reinterpret_cast<uint32_t*>(p + 2 * arr);
    uint32_t* idx_out = reinterpret_cast<uint32_t*>(p + 3 * arr);
    size_t temp = scratch_bytes - 4 * arr;
    const unsigned int kg = static_cast<unsigned int>((n + 255) / 256);
    direction_key_kernel<In><<<kg, 256, 0, stream>>>(dx, dy, dz, dq, n,
                                                     keys_in, idx_in);
    DPROP_CUDA(cudaGetLastError());
    DPROP_CUDA(cub::DeviceRadixSort::SortPairs(
        p + 4 * arr, temp, keys_in, keys_out, idx_in, idx_out,
        static_cast<int>(n), 0, 20, stream));
    *order = idx_out;
    return DPROP_OK;
}

dprop_status enqueue_direction_sort(const float* dx, const float* dy,
                                    const float* dz, const float* dq,
                                    uint64_t n, void* scratch,
                                    size_t scratch_bytes, cudaStream_t stream,
                                    const uint32_t** order) {
    return enqueue_sort<float>(dx, dy, dz, dq, n, scratch, scratch_bytes,
                               stream, order);
}

dprop_status enqueue_direction_sort(const double* dx, const double* dy,
                                    const double* dz, const double* dq,
                                    uint64_t n, void* scratch,
                                    size_t scratch_bytes, cudaStream_t stream,
                                    const uint32_t** order) {
    return enqueue_sort<double>(dx, dy, dz, dq, n, scratch, scratch_bytes,
                                stream, order);
}

}  // namespace dprop::api

using dprop::api::occupancy_of;
using dprop::api::sort_scratch_bytes;

namespace {

// The plain kernel for a detector: without the wire-surface code unless the
// detector needs it.  With the field gradient (use_field_gradient) the
// kernel carries the 18 position-column entries of the transport Jacobian;
// it is built for one register budget (8 CTAs per SM, 64 registers).
template <typename In, int MB>
void launch_plain_mb(int block, cudaStream_t st, const dprop_detector* det,
                     const field_view<float>& field, const prop_cfg<float>& cfg,
                     const io_ptrs<In>& io, uint64_t n, const uint32_t* order) {
    const unsigned int grid =
        static_cast<unsigned int>((n + block - 1) / block);
    if (cfg.step.field_gradient) {
        if (det->wires) {
            propagate_plain_kernel<In, 8, true, true>
                <<<grid, block, 0, st>>>(det->view_as<true>(), field, cfg, io,
                                         n, order);
        } else {
            propagate_plain_kernel<In, 8, false, true>
                <<<grid, block, 0, st>>>(det->view_as<false>(), field, cfg,
                                         io, n, order);
        }
        return;
    }
    if (det->wires) {
        propagate_plain_kernel<In, MB, true><<<grid, block, 0, st>>>(
            det->view_as<true>(), field, cfg, io, n, order);
    } else {
        propagate_plain_kernel<In, MB, false><<<grid, block, 0, st>>>(
            det->view_as<false>(), field, cfg, io, n, order);
    }
}

// Threads per CTA of a plain launch: dprop_launch.block_size, a multiple of
// 32 up to k_plain_max_block (0: k_plain_block); -1 if invalid.
int plain_block_of(const dprop_launch* lc) {
    const uint32_t b = lc ? lc->block_size : 0u;
    if (b == 0u) {
        return k_plain_block;
    }
    if (b % 32u != 0u || b > static_cast<uint32_t>(k_plain_max_block)) {
        return -1;
    }
    return static_cast<int>(b);
}

// The plain kernel at the launch's register budget and block size.
template <typename In>
dprop_status launch_plain(const dprop_launch* lc, cudaStream_t st,
                          const dprop_detector* det,
                          const field_view<float>& field,
                          const prop_cfg<float>& cfg, const io_ptrs<In>& io,
                          uint64_t n, const uint32_t* order) {
    const int block = plain_block_of(lc);
    if (block < 0) {
        return fail(DPROP_E_INVALID,
                    "plain method: block_size must be a multiple of 32 up to "
                    "256");
    }
    const int mb = occupancy_of(lc);
    if (mb == 8) {
        launch_plain_mb<In, 8>(block, st, det, field, cfg, io, n, order);
    } else if (mb == 16) {
        launch_plain_mb<In, 16>(block, st, det, field, cfg, io, n, order);
    } else {
        launch_plain_mb<In, 12>(block, st, det, field, cfg, io, n, order);
    }
    DPROP_CUDA(cudaGetLastError());
    return DPROP_OK;
}

// Scratch one propagation launch needs besides inputs and outputs.
struct launch_scratch {
    void* sort{nullptr};        // sort keys/indices + radix-sort temp storage
    size_t sort_bytes{0};
    void* rounds{nullptr};      // persistent method: track slots and queues
    size_t rounds_bytes{0};
};

// Enqueue one propagation on a stream using the given scratch; contains no
// allocation and no synchronisation, so it can be captured into a graph.
template <typename In>
dprop_status enqueue_propagation(const dprop_config& c,
                                 const dprop_launch* launch_cfg,
                                 const dprop_detector* det,
                                 const dprop_field* field,
                                 const io_ptrs<In>& io, uint64_t n,
                                 cudaStream_t stream,
                                 const launch_scratch& scr) {
    const prop_cfg<float> cfg = make_prop_cfg<float>(c);
    const uint32_t method = launch_cfg ? launch_cfg->method : DPROP_METHOD_PLAIN;
    const uint32_t* order = nullptr;
    if (launch_cfg && launch_cfg->sort_tracks) {
        const dprop_status s = dprop::api::enqueue_sort<In>(
            io.trk[4], io.trk[5], io.trk[6], io.trk[7], n, scr.sort,
            scr.sort_bytes,
            stream, &order);
        if (s != DPROP_OK) {
            return s;
        }
    }
    if (method == DPROP_METHOD_PERSISTENT) {
        return dprop::api::enqueue_rounds<In>(launch_cfg, det, field, cfg, io,
                                              n, order, scr.rounds,
                                              scr.rounds_bytes, stream);
    }
    return launch_plain<In>(launch_cfg, stream, det, field->view, cfg, io, n,
                            order);
}

// ------------------------------------------------------------ CUDA graphs
// With dprop_launch.use_graph the whole propagate call (key kernel, radix
// sort, propagation kernel) is captured once into a CUDA graph and replayed
// on later calls with the same arguments.  Each cached graph owns its
// scratch, so a replay never depends on the shared grow-only scratch.
struct graph_entry {
    std::vector<unsigned char> key;
    cudaGraphExec_t exec{nullptr};
    void* scratch{nullptr};
    uint64_t last_use{0};
    int device{0};
};
constexpr size_t k_graph_cache = 8;
std::vector<graph_entry> g_graphs;
uint64_t g_graph_clock = 0;
std::mutex g_graph_mutex;

void destroy_entry(graph_entry& e) {
    int cur = 0;
    const bool other = cudaGetDevice(&cur) == cudaSuccess && cur != e.device;
    if (other) {
        cudaSetDevice(e.device);
    }
    if (e.exec) {
        cudaGraphExecDestroy(e.exec);
    }
    if (e.scratch) {
        cudaFree(e.scratch);
    }
    e.exec = nullptr;
    e.scratch = nullptr;
    if (other) {
        cudaSetDevice(cur);
    }
}

template <typename In>
dprop_status launch(const dprop_config& c, const dprop_launch* launch_cfg,
                    const dprop_detector* det, const dprop_field* field,
                    const io_ptrs<In>& io, uint64_t n, cudaStream_t stream) {
    if (n == 0) {
        return DPROP_OK;
    }
    const bool sort = launch_cfg && launch_cfg->sort_tracks;
    const bool persistent = launch_cfg && launch_cfg->method == DPROP_METHOD_PERSISTENT;
    const uint32_t rec_cap =
        dprop::api::staged_capacity(make_prop_cfg<float>(c), io);
    if (!(launch_cfg && launch_cfg->use_graph)) {
        launch_scratch scr{};
        if (sort) {
            const size_t need = sort_scratch_bytes(n);
            if (g_sort.bytes < need) {
                if (g_sort.buf) {
                    DPROP_CUDA(cudaStreamSynchronize(stream));
                    cudaFree(g_sort.buf);
                    g_sort.buf = nullptr;
                    g_sort.bytes = 0;
                }
                DPROP_CUDA(cudaMalloc(&g_sort.buf, need));
                g_sort.bytes = need;
            }
            scr.sort = g_sort.buf;
            scr.sort_bytes = need;
        }
        if (persistent) {
            const size_t need =
                dprop::api::rounds_scratch_bytes(n, det->wires, rec_cap);
            if (g_rounds.bytes < need) {
                if (g_rounds.buf) {
                    DPROP_CUDA(cudaStreamSynchronize(stream));
                    cudaFree(g_rounds.buf);
                    g_rounds.buf = nullptr;
                    g_rounds.bytes = 0;
                }
                DPROP_CUDA(cudaMalloc(&g_rounds.buf, need));
                g_rounds.bytes = need;
            }
            scr.rounds = g_rounds.buf;
            scr.rounds_bytes = g_rounds.bytes;
        }
        return enqueue_propagation<In>(c, launch_cfg, det, field, io, n, stream,
                                       scr);
    }

    // graph path: key = everything the captured work depends on
    std::vector<unsigned char> key;
    auto put = [&key](const void* p, size_t b) {
        const unsigned char* q = static_cast<const unsigned char*>(p);
        key.insert(key.end(), q, q + b);
    };
    const int in_bytes = sizeof(In);
    put(&in_bytes, sizeof(in_bytes));
    put(&c, sizeof(c));
    put(launch_cfg, sizeof(*launch_cfg));
    put(&det, sizeof(det));
    put(&field, sizeof(field));
    put(&io, sizeof(io));
    put(&n, sizeof(n));
    int dev = 0;
    DPROP_CUDA(cudaGetDevice(&dev));
    put(&dev, sizeof(dev));

    std::lock_guard<std::mutex> lock(g_graph_mutex);
    for (graph_entry& e : g_graphs) {
        if (e.key == key) {
            e.last_use = ++g_graph_clock;
            DPROP_CUDA(cudaGraphLaunch(e.exec, stream));
            return DPROP_OK;
        }
    }
    graph_entry e;
    e.key = key;
    e.device = dev;
    const size_t sort_bytes = sort ? sort_scratch_bytes(n) : 0;
    const size_t rounds_bytes =
        persistent ? dprop::api::rounds_scratch_bytes(n, det->wires, rec_cap)
                   : 0;
    // The radix sort's temporary size carries the sort's alignment padding
    // and is usually odd: the persistent method's arrays after it start at
    // the next 256-byte boundary (an atomic on an unaligned word is a device
    // fault).
    const size_t rounds_offset = (sort_bytes + 255) & ~size_t(255);
    DPROP_CUDA(cudaMalloc(&e.scratch, rounds_offset + rounds_bytes + 256));
    launch_scratch scr{};
    scr.sort = e.scratch;
    scr.sort_bytes = sort_bytes;
    scr.rounds = static_cast<char*>(e.scratch) + rounds_offset;
    scr.rounds_bytes = rounds_bytes;
    cudaStream_t cap = nullptr;
    DPROP_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    DPROP_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    const dprop_status es =
        enqueue_propagation<In>(c, launch_cfg, det, field, io, n, cap, scr);
    const cudaError_t ce = cudaStreamEndCapture(cap, &graph);
    cudaStreamDestroy(cap);
    if (es != DPROP_OK || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaFree(e.scratch);
        return es != DPROP_OK ? es : cuda_fail(ce, "cudaStreamEndCapture");
    }
    const cudaError_t ie = cudaGraphInstantiate(&e.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        cudaFree(e.scratch);
        return cuda_fail(ie, "cudaGraphInstantiate");
    }
    if (g_graphs.size() >= k_graph_cache) {
        size_t oldest = 0;
        for (size_t i = 1; i < g_graphs.size(); ++i) {
            if (g_graphs[i].last_use < g_graphs[oldest].last_use) oldest = i;
        }
        destroy_entry(g_graphs[oldest]);
        g_graphs.erase(g_graphs.begin() + static_cast<long>(oldest));
    }
    e.last_use = ++g_graph_clock;
    g_graphs.push_back(e);
    DPROP_CUDA(cudaGraphLaunch(g_graphs.back().exec, stream));
    return DPROP_OK;
}

dprop_status check_config(const dprop_config* cfg) {
    if (!cfg) {
        return fail(DPROP_E_INVALID, "config is NULL");
    }
    if (cfg->max_iterations == 0u) {
        return fail(DPROP_E_INVALID, "max_iterations must be > 0");
    }
    return DPROP_OK;
}


// ------------------------------------------------ host path, jagged records
// dprop_propagate_host with results->rec_offsets: the batch is processed in
// chunks on two streams so that the host-to-device copy of one chunk, the
// propagation of another and the device-to-host copy of a third overlap.
// Each chunk's records are packed track by track (offsets from an exclusive
// scan of the per-track record counts) and only the stored records are
// copied back.

// per-track record count, clamped to the capacity; entry n is 0 so that an
// exclusive scan over n + 1 entries ends with the total
__global__ void clamp_counts_kernel(const uint32_t* __restrict__ n_rec,
                                    uint32_t cap, uint32_t n,
                                    uint32_t* __restrict__ counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const uint32_t c = n_rec[i];
        counts[i] = c < cap ? c : cap;
    } else if (i == n) {
        counts[i] = 0u;
    }
}

// Host pipeline shape: compute streams (chunks in flight) and the number of
// chunks a batch is split into.
#ifndef DPROP_PIPE_SLOTS
#define DPROP_PIPE_SLOTS 4
#endif
#ifndef DPROP_PIPE_SPLIT
#define DPROP_PIPE_SPLIT 4u
#endif
// Chunks whose propagation may run at the same time (0: all in flight).
#ifndef DPROP_PIPE_DEPTH
#define DPROP_PIPE_DEPTH 0
#endif
// Persistent method: chunk k + 1 starts its rounds once chunk k has run
// this many rounds (0: all chunks start together).  Started together, the
// chunks' rounds interleave and all chunks finish near the end of the batch,
// so the record copies start late (1 M toy tracks in 4 chunks on B200: the
// first chunk done after 21.8 ms, copies until 46.7 ms); started 16 rounds
// apart, the first chunk's records cross PCIe while the later chunks
// propagate in the earlier ones' tails (first chunk done after 16.5 ms,
// copies until 39.8 ms).  One chunk after the other costs each chunk the
// method's per-round latency (48 ms end to end).
#ifndef DPROP_PIPE_STAGGER
#define DPROP_PIPE_STAGGER 16
#endif

struct record_arrays {
    uint64_t* barcode;
    float* bound[6];
    float* cov[21];
    float* path;
    uint8_t* flags;
};

// slot-major records (k * n + t) -> packed records (offset[t] + k)
__global__ void pack_records_kernel(record_arrays src, record_arrays dst,
                                    const uint32_t* __restrict__ counts,
                                    const uint32_t* __restrict__ offsets,
                                    uint32_t n) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) {
        return;
    }
    const uint32_t m = counts[t];
    const uint32_t o = offsets[t];
    for (uint32_t k = 0; k < m; ++k) {
        const uint64_t si = static_cast<uint64_t>(k) * n + t;
        const uint64_t di = static_cast<uint64_t>(o) + k;
        if (dst.barcode) dst.barcode[di] = src.barcode[si];
        for (int i = 0; i < 6; ++i) {
            if (dst.bound[i]) dst.bound[i][di] = src.bound[i][si];
        }
        for (int i = 0; i < 21; ++i) {
            if (dst.cov[i]) dst.cov[i][di] = src.cov[i][si];
        }
        if (dst.path) dst.path[di] = src.path[si];
        if (dst.flags) dst.flags[di] = src.flags[si];
    }
}

// One pipeline slot: a compute stream (inputs in, sort, propagation, record
// packing, per-track outputs out) and its device buffers.  The packed
// records of all slots drain on one copy stream, in chunk order, so that the
// next chunks' propagation does not queue behind the record copies.  At most
// k_pipe_slots compute streams plus the copy stream stay within the device's
// default eight hardware work queues, so that a copy does not wait behind an
// unrelated kernel sharing its queue.
struct pipe_slot {
    cudaStream_t stream{nullptr};
    cudaEvent_t counted{nullptr};   // packed records and offsets ready
    cudaEvent_t drained{nullptr};   // packed records copied out
    cudaEvent_t ran{nullptr};       // propagation and packing done
    cudaEvent_t mark{nullptr};      // persistent method: the chunk's rounds
                                    // reached DPROP_PIPE_STAGGER
    void* dev{nullptr};
    size_t dev_bytes{0};
    uint32_t* host_offsets{nullptr};  // pinned, chunk + 1 entries
    size_t host_entries{0};
};
constexpr int k_pipe_slots = DPROP_PIPE_SLOTS;
pipe_slot g_pipe[k_pipe_slots];
cudaStream_t g_copy_stream = nullptr;

dprop_status ensure_pipe(pipe_slot& ps, int index, size_t dev_bytes,
                         size_t chunk) {
    if (!ps.stream) {
        // earlier chunks of a batch run at higher priority: the block
        // scheduler finishes them first, so that their records start crossing
        // PCIe early, while later chunks fill the SMs their tails leave idle
        int least = 0, greatest = 0;
        DPROP_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        const int prio = (greatest + index < least) ? greatest + index : least;
        DPROP_CUDA(cudaStreamCreateWithPriority(&ps.stream,
                                                cudaStreamNonBlocking, prio));
        if (!g_copy_stream) {
            DPROP_CUDA(cudaStreamCreateWithFlags(&g_copy_stream,
                                                 cudaStreamNonBlocking));
        }
        DPROP_CUDA(cudaEventCreateWithFlags(&ps.counted, cudaEventDisableTiming));
        DPROP_CUDA(cudaEventCreateWithFlags(&ps.drained, cudaEventDisableTiming));
        DPROP_CUDA(cudaEventCreateWithFlags(&ps.ran, cudaEventDisableTiming));
        DPROP_CUDA(cudaEventCreateWithFlags(&ps.mark, cudaEventDisableTiming));
        // nothing to wait for before the first packing
        DPROP_CUDA(cudaEventRecord(ps.drained, g_copy_stream));
    }
    if (ps.dev_bytes < dev_bytes) {
        if (ps.dev) {
            cudaFree(ps.dev);
            ps.dev = nullptr;
            ps.dev_bytes = 0;
        }
        DPROP_CUDA(cudaMalloc(&ps.dev, dev_bytes));
        ps.dev_bytes = dev_bytes;
    }
    if (ps.host_entries < chunk + 1) {
        if (ps.host_offsets) {
            cudaFreeHost(ps.host_offsets);
            ps.host_offsets = nullptr;
        }
        DPROP_CUDA(cudaMallocHost(reinterpret_cast<void**>(&ps.host_offsets),
                                  (chunk + 1) * sizeof(uint32_t)));
        ps.host_entries = chunk + 1;
    }
    return DPROP_OK;
}

// device buffers of one slot (the same carving for every chunk)
struct slot_buffers {
    const double* trk[8];
    dprop_results dr;
    record_arrays slotm, packed;
    uint32_t *counts, *offsets, *keys_in, *keys_out, *idx_in, *idx_out;
    void* sort_tmp;
    void* scan_tmp;
};

size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

slot_buffers carve_slot(void* base, uint64_t chunk, uint64_t rec_slot,
                        bool with_cov, size_t sort_temp, size_t scan_temp) {
    slot_buffers b{};
    char* p = static_cast<char*>(base);
    auto take = [&](size_t bytes) {
        char* r = p;
        p += al256(bytes);
        return r;
    };
    for (int i = 0; i < 8; ++i) {
        b.trk[i] = reinterpret_cast<double*>(take(chunk * sizeof(double)));
    }
    dprop_results& dr = b.dr;
    dr.status = reinterpret_cast<uint8_t*>(take(chunk));
    dr.n_records = reinterpret_cast<uint32_t*>(take(chunk * 4));
    dr.n_steps = reinterpret_cast<uint32_t*>(take(chunk * 4));
    dr.n_trials = reinterpret_cast<uint32_t*>(take(chunk * 4));
    dr.path_length = take(chunk * 4);
    dr.n_intersections = reinterpret_cast<uint32_t*>(take(chunk * 4));
    dr.n_transports = reinterpret_cast<uint32_t*>(take(chunk * 4));
    dr.n_material = reinterpret_cast<uint32_t*>(take(chunk * 4));
    for (int i = 0; i < 8; ++i) {
        dr.final_free[i] = take(chunk * 4);
    }
    b.slotm.barcode = reinterpret_cast<uint64_t*>(take(rec_slot * 8));
    b.packed.barcode = reinterpret_cast<uint64_t*>(take(rec_slot * 8));
    for (int i = 0; i < 6; ++i) {
        b.slotm.bound[i] = reinterpret_cast<float*>(take(rec_slot * 4));
        b.packed.bound[i] = reinterpret_cast<float*>(take(rec_slot * 4));
    }
    for (int i = 0; i < 21; ++i) {
        float* a = reinterpret_cast<float*>(take(rec_slot * 4));
        float* c = reinterpret_cast<float*>(take(rec_slot * 4));
        if (with_cov) {
            b.slotm.cov[i] = a;
            b.packed.cov[i] = c;
        }
    }
    b.slotm.path = reinterpret_cast<float*>(take(rec_slot * 4));
    b.packed.path = reinterpret_cast<float*>(take(rec_slot * 4));
    b.slotm.flags = reinterpret_cast<uint8_t*>(take(rec_slot));
    b.packed.flags = reinterpret_cast<uint8_t*>(take(rec_slot));
    dr.rec_barcode = b.slotm.barcode;
    for (int i = 0; i < 6; ++i) dr.rec_bound[i] = b.slotm.bound[i];
    for (int i = 0; i < 21; ++i) dr.rec_cov[i] = b.slotm.cov[i];
    dr.rec_path = b.slotm.path;
    dr.rec_flags = b.slotm.flags;
    b.counts = reinterpret_cast<uint32_t*>(take((chunk + 1) * 4));
    b.offsets = reinterpret_cast<uint32_t*>(take((chunk + 1) * 4));
    b.keys_in = reinterpret_cast<uint32_t*>(take((chunk + 1) * 4));
    b.keys_out = reinterpret_cast<uint32_t*>(take((chunk + 1) * 4));
    b.idx_in = reinterpret_cast<uint32_t*>(take((chunk + 1) * 4));
    b.idx_out = reinterpret_cast<uint32_t*>(take((chunk + 1) * 4));
    b.sort_tmp = take(sort_temp);
    b.scan_tmp = take(scan_temp);
    return b;
}

dprop_status propagate_host_jagged(const dprop_config& c,
                                   const dprop_launch* lc,
                                   const dprop_detector* det,
                                   const dprop_field* field,
                                   const dprop_tracks& tracks,
                                   const dprop_results& out, uint64_t n) {
    const uint64_t cap = c.max_records;
    // about k_pipe_slots chunks per batch, 32 Ki - 256 Ki tracks each
    uint64_t chunk = ((n / DPROP_PIPE_SPLIT + 1023u) / 1024u) * 1024u;
    chunk = chunk < 32768u ? 32768u : (chunk > 262144u ? 262144u : chunk);
    chunk = n < chunk ? n : chunk;
    const uint64_t n_chunks = (n + chunk - 1u) / chunk;
    const int n_slots = n_chunks < static_cast<uint64_t>(k_pipe_slots)
                            ? static_cast<int>(n_chunks)
                            : k_pipe_slots;
    const prop_cfg<float> pcfg = make_prop_cfg<float>(c);
    const bool sort = (lc == nullptr) || lc->sort_tracks != 0u;
    const void* h_trk[8] = {tracks.pos[0], tracks.pos[1], tracks.pos[2],
                            tracks.time,   tracks.dir[0], tracks.dir[1],
                            tracks.dir[2], tracks.qop};
    for (int i = 0; i < 8; ++i) {
        if (!h_trk[i]) {
            return fail(DPROP_E_INVALID, "propagate_host: missing track array");
        }
    }
    bool with_cov = false;
    for (int i = 0; i < 21; ++i) {
        with_cov = with_cov || out.rec_cov[i] != nullptr;
    }

    // device scratch layout of one pipeline slot
    size_t sort_temp = 0, scan_temp = 0;
    DPROP_CUDA(cub::DeviceRadixSort::SortPairs(
        nullptr, sort_temp, static_cast<const uint32_t*>(nullptr),
        static_cast<uint32_t*>(nullptr), static_cast<const uint32_t*>(nullptr),
        static_cast<uint32_t*>(nullptr), static_cast<int>(chunk), 0, 20));
    DPROP_CUDA(cub::DeviceScan::ExclusiveSum(
        nullptr, scan_temp, static_cast<const uint32_t*>(nullptr),
        static_cast<uint32_t*>(nullptr), static_cast<int>(chunk + 1)));
    const size_t rec_slot = cap * chunk;
    size_t need = 0;
    need += 8 * al256(chunk * sizeof(double));                        // inputs
    need += al256(chunk) + 7 * al256(chunk * 4) + 8 * al256(chunk * 4);  // per-track
    need += 2 * (al256(rec_slot * 8) + 28 * al256(rec_slot * 4) + al256(rec_slot));
    need += 6 * al256((chunk + 1) * 4) + al256(sort_temp) + al256(scan_temp);
    const bool rounds = lc && lc->method == DPROP_METHOD_PERSISTENT;
    const size_t rounds_bytes =
        rounds ? al256(dprop::api::rounds_scratch_bytes(
                     chunk, det->wires, static_cast<uint32_t>(cap)))
               : 0;
    need += rounds_bytes;
    for (int k = 0; k < n_slots; ++k) {
        const dprop_status s = ensure_pipe(g_pipe[k], k, need, chunk);
        if (s != DPROP_OK) {
            return s;
        }
    }
    auto carve = [&](int sl) {
        return carve_slot(g_pipe[sl].dev, chunk, rec_slot, with_cov, sort_temp,
                          scan_temp);
    };
    // the persistent method's slot arrays and queues: the tail of the block
    auto rounds_scratch = [&](int sl) {
        return static_cast<char*>(g_pipe[sl].dev) + (need - rounds_bytes);
    };
    cudaEvent_t inputs_ready = nullptr;
    DPROP_CUDA(cudaEventCreateWithFlags(&inputs_ready, cudaEventDisableTiming));
    // make the pipeline streams wait for work already queued on the legacy
    // stream (e.g. the caller's uploads)
    DPROP_CUDA(cudaEventRecord(inputs_ready, 0));
    for (int k = 0; k < n_slots; ++k) {
        DPROP_CUDA(cudaStreamWaitEvent(g_pipe[k].stream, inputs_ready, 0));
    }

    struct chunk_info {
        uint64_t begin;
        uint64_t count;
        record_arrays packed;
    };
    uint64_t rec_base = 0;

    // copy a finished chunk's packed records into the caller's arrays (on
    // the copy stream; the host has seen the chunk's record count)
    auto drain = [&](const chunk_info& ci, int sl) -> dprop_status {
        pipe_slot& ps = g_pipe[sl];
        DPROP_CUDA(cudaEventSynchronize(ps.counted));
        const uint32_t total = ps.host_offsets[ci.count];
        for (uint64_t t = 0; t < ci.count; ++t) {
            out.rec_offsets[ci.begin + t] = rec_base + ps.host_offsets[t];
        }
        auto d2h = [&](void* h, const void* d, size_t elem) -> dprop_status {
            if (h && d && total) {
                DPROP_CUDA(cudaMemcpyAsync(static_cast<char*>(h) + rec_base * elem,
                                           d, total * elem,
                                           cudaMemcpyDeviceToHost,
                                           g_copy_stream));
            }
            return DPROP_OK;
        };
        dprop_status s = DPROP_OK;
        if ((s = d2h(out.rec_barcode, ci.packed.barcode, 8)) != DPROP_OK) return s;
        for (int i = 0; i < 6; ++i) {
            if ((s = d2h(out.rec_bound[i], ci.packed.bound[i], 4)) != DPROP_OK) return s;
        }
        for (int i = 0; i < 21; ++i) {
            if ((s = d2h(out.rec_cov[i], ci.packed.cov[i], 4)) != DPROP_OK) return s;
        }
        if ((s = d2h(out.rec_path, ci.packed.path, 4)) != DPROP_OK) return s;
        if ((s = d2h(out.rec_flags, ci.packed.flags, 1)) != DPROP_OK) return s;
        DPROP_CUDA(cudaEventRecord(ps.drained, g_copy_stream));
        rec_base += total;
        return DPROP_OK;
    };

    // inputs in and direction sort of one chunk
    auto stage_in = [&](uint64_t begin, uint64_t m, int sl) -> dprop_status {
        const cudaStream_t st = g_pipe[sl].stream;
        const slot_buffers b = carve(sl);
        for (int i = 0; i < 8; ++i) {
            DPROP_CUDA(cudaMemcpyAsync(const_cast<double*>(b.trk[i]),
                                       static_cast<const double*>(h_trk[i]) + begin,
                                       m * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        if (sort) {
            const unsigned int kg = static_cast<unsigned int>((m + 255) / 256);
            direction_key_kernel<double><<<kg, 256, 0, st>>>(
                b.trk[4], b.trk[5], b.trk[6], b.trk[7], m, b.keys_in, b.idx_in);
            size_t tb = sort_temp;
            DPROP_CUDA(cub::DeviceRadixSort::SortPairs(
                b.sort_tmp, tb, b.keys_in, b.keys_out, b.idx_in, b.idx_out,
                static_cast<int>(m), 0, 20, st));
        }
        return DPROP_OK;
    };

    // propagation, record packing and per-track outputs of one chunk; with
    // a pipeline depth d, chunk k propagates after chunk k - d has; with
    // the persistent method chunk k starts DPROP_PIPE_STAGGER rounds after
    // chunk k - 1
    uint64_t n_run = 0;
    int run_slot[k_pipe_slots] = {};
    auto stage_run = [&](uint64_t begin, uint64_t m, int sl) -> dprop_status {
        pipe_slot& ps = g_pipe[sl];
        const cudaStream_t st = ps.stream;
        const slot_buffers b = carve(sl);
        constexpr int depth = DPROP_PIPE_DEPTH;
        static_assert(depth < k_pipe_slots, "pipeline depth below the slots");
        if (depth > 0 && n_run >= static_cast<uint64_t>(depth)) {
            DPROP_CUDA(cudaStreamWaitEvent(
                st, g_pipe[run_slot[(n_run - depth) % k_pipe_slots]].ran, 0));
        }
        dprop_tracks dt{};
        for (int i = 0; i < 3; ++i) {
            dt.pos[i] = b.trk[i];
            dt.dir[i] = b.trk[4 + i];
        }
        dt.time = b.trk[3];
        dt.qop = b.trk[7];
        const io_ptrs<double> io = make_io<double>(dt, b.dr);
        if (rounds) {
            constexpr uint32_t stagger = DPROP_PIPE_STAGGER;
            if (stagger > 0u && n_run > 0u) {
                DPROP_CUDA(cudaStreamWaitEvent(
                    st, g_pipe[run_slot[(n_run - 1) % k_pipe_slots]].mark, 0));
            }
            const dprop_status s = dprop::api::enqueue_rounds<double>(
                lc, det, field, pcfg, io, m, sort ? b.idx_out : nullptr,
                rounds_scratch(sl), rounds_bytes, st,
                stagger > 0u ? ps.mark : nullptr, stagger);
            if (s != DPROP_OK) return s;
        } else {
            const dprop_status s = launch_plain<double>(
                lc, st, det, field->view, pcfg, io, m,
                sort ? b.idx_out : nullptr);
            if (s != DPROP_OK) return s;
        }
        DPROP_CUDA(cudaGetLastError());
        // pack the records
        const unsigned int cg = static_cast<unsigned int>((m + 1 + 255) / 256);
        clamp_counts_kernel<<<cg, 256, 0, st>>>(b.dr.n_records,
                                                static_cast<uint32_t>(cap),
                                                static_cast<uint32_t>(m), b.counts);
        size_t sb = scan_temp;
        DPROP_CUDA(cub::DeviceScan::ExclusiveSum(b.scan_tmp, sb, b.counts,
                                                 b.offsets,
                                                 static_cast<int>(m + 1), st));
        // the packed buffers are free once the slot's last drain finished
        DPROP_CUDA(cudaStreamWaitEvent(st, ps.drained, 0));
        const unsigned int pg = static_cast<unsigned int>((m + 127) / 128);
        pack_records_kernel<<<pg, 128, 0, st>>>(b.slotm, b.packed, b.counts,
                                                b.offsets,
                                                static_cast<uint32_t>(m));
        DPROP_CUDA(cudaGetLastError());
        DPROP_CUDA(cudaEventRecord(ps.ran, st));
        run_slot[n_run % k_pipe_slots] = sl;
        ++n_run;
        // per-track outputs and the offsets back to the host
        auto d2h = [&](void* h, const void* d, size_t elem) -> dprop_status {
            if (h && d) {
                DPROP_CUDA(cudaMemcpyAsync(static_cast<char*>(h) + begin * elem, d,
                                           m * elem, cudaMemcpyDeviceToHost, st));
            }
            return DPROP_OK;
        };
        const dprop_results& dr = b.dr;
        dprop_status s = DPROP_OK;
        if ((s = d2h(out.status, dr.status, 1)) != DPROP_OK) return s;
        if ((s = d2h(out.n_records, dr.n_records, 4)) != DPROP_OK) return s;
        if ((s = d2h(out.n_steps, dr.n_steps, 4)) != DPROP_OK) return s;
        if ((s = d2h(out.n_trials, dr.n_trials, 4)) != DPROP_OK) return s;
        if ((s = d2h(out.path_length, dr.path_length, 4)) != DPROP_OK) return s;
        if ((s = d2h(out.n_intersections, dr.n_intersections, 4)) != DPROP_OK) return s;
        if ((s = d2h(out.n_transports, dr.n_transports, 4)) != DPROP_OK) return s;
        if ((s = d2h(out.n_material, dr.n_material, 4)) != DPROP_OK) return s;
        for (int i = 0; i < 8; ++i) {
            if ((s = d2h(out.final_free[i], dr.final_free[i], 4)) != DPROP_OK) return s;
        }
        DPROP_CUDA(cudaMemcpyAsync(ps.host_offsets, b.offsets, (m + 1) * 4,
                                   cudaMemcpyDeviceToHost, st));
        DPROP_CUDA(cudaEventRecord(ps.counted, st));
        return DPROP_OK;
    };

    // the chunk each slot still has to drain (drained in chunk order: the
    // slots are used round robin)
    chunk_info pending[k_pipe_slots] = {};
    bool has_pending[k_pipe_slots] = {};
    int slot = 0;
    // waves of n_slots chunks: first every chunk's inputs and sort, then the
    // propagation kernels, so that no sort waits behind a propagation kernel
    // that holds the SMs' registers
    const uint64_t wave = chunk * static_cast<uint64_t>(n_slots);
    for (uint64_t w0 = 0; w0 < n; w0 += wave) {
        const uint64_t w1 = (n - w0) < wave ? n : w0 + wave;
        int sl = slot;
        for (uint64_t begin = w0; begin < w1;
             begin += chunk, sl = (sl + 1) % n_slots) {
            const uint64_t m = (w1 - begin) < chunk ? (w1 - begin) : chunk;
            if (has_pending[sl]) {
                const dprop_status s = drain(pending[sl], sl);
                if (s != DPROP_OK) return s;
                has_pending[sl] = false;
            }
            const dprop_status s = stage_in(begin, m, sl);
            if (s != DPROP_OK) return s;
        }
        sl = slot;
        for (uint64_t begin = w0; begin < w1;
             begin += chunk, sl = (sl + 1) % n_slots) {
            const uint64_t m = (w1 - begin) < chunk ? (w1 - begin) : chunk;
            const dprop_status s = stage_run(begin, m, sl);
            if (s != DPROP_OK) return s;
            pending[sl] = chunk_info{begin, m, carve(sl).packed};
            has_pending[sl] = true;
        }
        slot = sl;
    }
    // drain what is left, oldest chunk first
    for (int k = 0; k < n_slots; ++k) {
        const int sl = (slot + k) % n_slots;
        if (has_pending[sl]) {
            const dprop_status s = drain(pending[sl], sl);
            if (s != DPROP_OK) return s;
            has_pending[sl] = false;
        }
    }
    out.rec_offsets[n] = rec_base;
    for (int k = 0; k < n_slots; ++k) {
        DPROP_CUDA(cudaStreamSynchronize(g_pipe[k].stream));
    }
    DPROP_CUDA(cudaStreamSynchronize(g_copy_stream));
    cudaEventDestroy(inputs_ready);
    return DPROP_OK;
}

}  // namespace

// ====================================================================== ABI
extern "C" {

uint32_t dprop_abi_version(void) { return DPROP_ABI_VERSION; }

const char* dprop_last_error(void) { return g_last_error.c_str(); }

void dprop_config_default(dprop_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->min_stepsize = 1e-4f;
    c->rk_error_tol = 1e-4f;
    c->step_constraint = FLT_MAX;
    c->path_limit = 5000.f;
    c->max_rk_updates = 10000u;
    c->use_mean_loss = 1;
    c->use_eloss_gradient = 0;
    c->use_field_gradient = 0;
    c->do_covariance_transport = 1;
    c->min_mask_tolerance = 1e-5f;
    c->max_mask_tolerance = 3.f;
    c->mask_tolerance_scalor = 5e-2f;
    c->path_tolerance = 1e-3f;
    c->overstep_tolerance = -1.f;
    c->search_window[0] = 0u;
    c->search_window[1] = 0u;
    c->accumulated_error = 0.001f;
    c->n_scattering_stddev = 3;
    c->estimate_scattering_noise = 1;
    c->use_path_limit_aborter = 1;
    c->use_material_interactor = 1;
    c->record_all_surfaces = 0;
    // the reference's muon mass, a float product
    // (definitions/pdg_particle.hpp:84: 105.6583755f * unit<float>::MeV)
    c->mass = 105.6583755f * 1e-3f;
    c->pdg = 13;
    c->max_records = 32u;
    c->max_iterations = 200000u;
}

dprop_status dprop_detector_create(const dprop_detector_desc* d, int device,
                                   dprop_detector** out) {
    if (!d || !out) {
        return fail(DPROP_E_INVALID, "detector_create: NULL argument");
    }
    *out = nullptr;
    const std::string problem = validate_desc(d);
    if (!problem.empty()) {
        const bool unsupported = problem.find("not supported") != std::string::npos;
        return fail(unsupported ? DPROP_E_UNSUPPORTED : DPROP_E_INVALID,
                    "detector_create: " + problem);
    }
    const host_tables<float> t = convert_desc<float>(d);
    DPROP_CUDA(cudaSetDevice(device));
    auto* det = new dprop_detector();
    det->device = device;
    det->n_volumes = d->n_volumes;
    det->n_surfaces = d->n_surfaces;
    dprop_status st = DPROP_OK;
    if ((st = upload(t.volumes, &det->volumes)) != DPROP_OK ||
        (st = upload(t.surfaces, &det->surfaces)) != DPROP_OK ||
        (st = upload(t.masks, &det->masks)) != DPROP_OK ||
        (st = upload(t.transforms, &det->transforms)) != DPROP_OK ||
        (st = upload(t.slabs, &det->slabs)) != DPROP_OK ||
        (st = upload(t.bf_surfaces, &det->bf_surfaces)) != DPROP_OK ||
        (st = upload(t.grids, &det->grids)) != DPROP_OK ||
        (st = upload(t.grid_bins, &det->grid_bins)) != DPROP_OK ||
        (!t.vol_material.empty() &&
         (st = upload(t.vol_material, &det->vol_material)) != DPROP_OK)) {
        dprop_detector_destroy(det);
        return st;
    }
    det->wires = has_volume_material(d);
    for (uint32_t i = 0; i < d->n_surfaces; ++i) {
        det->wires = det->wires || d->surfaces[i].shape == DPROP_SHAPE_LINE ||
                     d->surfaces[i].material_kind != 0u;
    }
    for (uint32_t i = 0; i < d->n_slabs; ++i) {
        det->wires = det->wires || d->slabs[i].kind == DPROP_MATERIAL_ROD;
    }
    for (uint32_t i = 0; i < d->n_grids; ++i) {
        det->wires = det->wires || d->grids[i].multi != 0u;
    }
    const host_tables<double> td = convert_desc<double>(d);
    if ((st = upload(td.masks, &det->masks_d)) != DPROP_OK ||
        (st = upload(td.transforms, &det->transforms_d)) != DPROP_OK ||
        (st = upload(td.slabs, &det->slabs_d)) != DPROP_OK ||
        (st = upload(td.grids, &det->grids_d)) != DPROP_OK) {
        dprop_detector_destroy(det);
        return st;
    }
    *out = det;
    return DPROP_OK;
}

dprop_status dprop_detector_destroy(dprop_detector* det) {
    if (!det) {
        return DPROP_OK;
    }
    cudaFree(det->volumes);
    cudaFree(det->surfaces);
    cudaFree(det->masks);
    cudaFree(det->transforms);
    cudaFree(det->slabs);
    cudaFree(det->bf_surfaces);
    cudaFree(det->grids);
    cudaFree(det->grid_bins);
    cudaFree(det->vol_material);
    cudaFree(det->masks_d);
    cudaFree(det->transforms_d);
    cudaFree(det->slabs_d);
    cudaFree(det->grids_d);
    delete det;
    return DPROP_OK;
}

dprop_status dprop_autotune(const dprop_config* cfg, const dprop_detector* det,
                            const dprop_field* field, const dprop_tracks* tracks,
                            uint64_t n, dprop_launch* launch_out,
                            float* timings_ms, void* stream_ptr) {
    dprop_status s = check_config(cfg);
    if (s != DPROP_OK) {
        return s;
    }
    if (!det || !field || !tracks || !launch_out) {
        return fail(DPROP_E_INVALID, "autotune: NULL argument");
    }
    if (n == 0) {
        return DPROP_OK;
    }
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    // at most 2^20 tracks: the persistent method's per-round costs are
    // amortised over the batch, so a small sample would misjudge it
    const uint64_t m = n < 1048576u ? n : 1048576u;
    const uint64_t cap = cfg->max_records;
    // temporary results for the trial runs
    const size_t per_track = 1 + 6 * 4 + 8 * 4 + 16;
    const size_t per_rec = 8 + 6 * 4 + 21 * 4 + 4 + 1;
    void* buf = nullptr;
    DPROP_CUDA(cudaMalloc(&buf, m * per_track + cap * m * per_rec + 4096));
    char* p = static_cast<char*>(buf);
    auto take = [&](size_t b) {
        char* r = p;
        p += (b + 15) & ~size_t(15);
        return r;
    };
    dprop_results r{};
    r.status = reinterpret_cast<uint8_t*>(take(m));
    r.n_records = reinterpret_cast<uint32_t*>(take(4 * m));
    r.n_steps = reinterpret_cast<uint32_t*>(take(4 * m));
    r.n_trials = reinterpret_cast<uint32_t*>(take(4 * m));
    r.path_length = take(4 * m);
    r.rec_barcode = reinterpret_cast<uint64_t*>(take(8 * cap * m));
    for (int i = 0; i < 6; ++i) r.rec_bound[i] = take(4 * cap * m);
    for (int i = 0; i < 21; ++i) r.rec_cov[i] = take(4 * cap * m);
    r.rec_path = take(4 * cap * m);
    r.rec_flags = reinterpret_cast<uint8_t*>(take(cap * m));
    const io_ptrs<float> io = make_io<float>(*tracks, r);

    // plain: register budget (resident CTAs per SM) x block size x
    // direction sort; persistent: step-phase register budget x steps per
    // round x tracks per warp (yield lanes) x rounds x volume re-sort
    // interval x direction sort
    struct cand {
        uint32_t method, block, ctas, sort, steps, yield, rounds, interval;
    };
    const cand cands[DPROP_AUTOTUNE_CANDIDATES] = {
        {DPROP_METHOD_PLAIN, 128, 8, 1, 0, 0, 0, 0},
        {DPROP_METHOD_PLAIN, 128, 12, 1, 0, 0, 0, 0},
        {DPROP_METHOD_PLAIN, 128, 16, 1, 0, 0, 0, 0},
        {DPROP_METHOD_PLAIN, 256, 16, 1, 0, 0, 0, 0},
        {DPROP_METHOD_PLAIN, 128, 16, 0, 0, 0, 0, 0},
        {DPROP_METHOD_PERSISTENT, 128, 3, 1, 16, 16, 64, 0},
        {DPROP_METHOD_PERSISTENT, 128, 3, 1, 16, 16, 64, 1},
        {DPROP_METHOD_PERSISTENT, 128, 4, 1, 16, 16, 64, 0},
        {DPROP_METHOD_PERSISTENT, 128, 4, 1, 16, 16, 64, 2},
        {DPROP_METHOD_PERSISTENT, 128, 5, 1, 16, 16, 64, 0},
        {DPROP_METHOD_PERSISTENT, 128, 4, 1, 16, 8, 96, 0},
        {DPROP_METHOD_PERSISTENT, 128, 4, 1, 64, 12, 64, 0},
        {DPROP_METHOD_PERSISTENT, 128, 4, 0, 16, 16, 64, 0}};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 3.4e38f;
    int best_i = 1;
    for (int i = 0; i < DPROP_AUTOTUNE_CANDIDATES && s == DPROP_OK; ++i) {
        dprop_launch lc{};
        lc.use_graph = launch_out->use_graph;
        lc.method = cands[i].method;
        lc.block_size = cands[i].block;
        lc.sort_interval = cands[i].interval;
        lc.ctas_per_sm = cands[i].ctas;
        lc.sort_tracks = cands[i].sort;
        lc.steps_per_round = cands[i].steps;
        lc.yield_lanes = cands[i].yield;
        lc.rounds = cands[i].rounds;
        s = launch<float>(*cfg, &lc, det, field, io, m, stream);  // warm-up
        if (s != DPROP_OK) break;
        cudaEventRecord(e0, stream);
        for (int k = 0; k < 2 && s == DPROP_OK; ++k) {
            s = launch<float>(*cfg, &lc, det, field, io, m, stream);
        }
        cudaEventRecord(e1, stream);
        const cudaError_t ce = cudaEventSynchronize(e1);
        if (ce != cudaSuccess) {
            s = cuda_fail(ce, "autotune");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms *= 0.5f;
        if (timings_ms) timings_ms[i] = ms;
        if (ms < best) {
            best = ms;
            best_i = i;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    if (s != DPROP_OK) {
        return s;
    }
    launch_out->method = cands[best_i].method;
    launch_out->block_size = cands[best_i].block;
    launch_out->sort_interval = cands[best_i].interval;
    launch_out->ctas_per_sm = cands[best_i].ctas;
    launch_out->sort_tracks = cands[best_i].sort;
    launch_out->steps_per_round = cands[best_i].steps;
    launch_out->yield_lanes = cands[best_i].yield;
    launch_out->rounds = cands[best_i].rounds;
    return DPROP_OK;
}

dprop_status dprop_detector_info(const dprop_detector* det, uint32_t* n_volumes,
                                 uint32_t* n_surfaces) {
    if (!det) {
        return fail(DPROP_E_INVALID, "detector_info: NULL detector");
    }
    if (n_volumes) *n_volumes = det->n_volumes;
    if (n_surfaces) *n_surfaces = det->n_surfaces;
    return DPROP_OK;
}

dprop_status dprop_field_create_const(double bx, double by, double bz,
                                      int device, dprop_field** out) {
    if (!out) {
        return fail(DPROP_E_INVALID, "field_create_const: NULL out");
    }
    auto* f = new dprop_field();
    f->device = device;
    f->view.kind = 0u;
    f->view.n_r = f->view.n_phi = f->view.n_z = 1u;
    f->view.b[0] = static_cast<float>(bx);
    f->view.b[1] = static_cast<float>(by);
    f->view.b[2] = static_cast<float>(bz);
    f->view.nodes = nullptr;
    f->view_d.kind = 0u;
    f->view_d.n_r = f->view_d.n_phi = f->view_d.n_z = 1u;
    f->view_d.b[0] = bx;
    f->view_d.b[1] = by;
    f->view_d.b[2] = bz;
    f->view_d.nodes = nullptr;
    *out = f;
    return DPROP_OK;
}

dprop_status dprop_field_create_grid(const double* lo, const double* hi,
                                     const uint32_t* n, const float* values,
                                     int device, dprop_field** out) {
    if (!lo || !hi || !n || !values || !out) {
        return fail(DPROP_E_INVALID, "field_create_grid: NULL argument");
    }
    if (n[0] == 0 || n[1] == 0 || n[2] == 0 || (n[0] > 1 && !(hi[0] > lo[0])) ||
        (n[2] > 1 && !(hi[2] > lo[2]))) {
        return fail(DPROP_E_INVALID, "field_create_grid: bad axes");
    }
    const uint64_t nodes = static_cast<uint64_t>(n[0]) * n[1] * n[2];
    std::vector<float4> h(nodes);
    for (uint64_t i = 0; i < nodes; ++i) {
        h[i] = make_float4(values[3 * i], values[3 * i + 1], values[3 * i + 2], 0.f);
    }
    DPROP_CUDA(cudaSetDevice(device));
    auto* f = new dprop_field();
    f->device = device;
    dprop_status st = upload(h, &f->nodes);
    if (st != DPROP_OK) {
        delete f;
        return st;
    }
    field_view<float>& v = f->view;
    v.kind = 1u;
    v.n_r = n[0];
    v.n_phi = n[1];
    v.n_z = n[2];
    v.b[0] = v.b[1] = v.b[2] = 0.f;
    v.r_lo = static_cast<float>(lo[0]);
    v.r_step_inv = n[0] > 1 ? static_cast<float>((n[0] - 1) / (hi[0] - lo[0])) : 0.f;
    v.phi_lo = static_cast<float>(lo[1]);
    v.phi_step_inv = static_cast<float>(n[1] / (2.0 * constant::pi));
    v.z_lo = static_cast<float>(lo[2]);
    v.z_step_inv = n[2] > 1 ? static_cast<float>((n[2] - 1) / (hi[2] - lo[2])) : 0.f;
    v.nodes = f->nodes;
    field_view<double>& vd = f->view_d;
    vd.kind = 1u;
    vd.n_r = n[0];
    vd.n_phi = n[1];
    vd.n_z = n[2];
    vd.b[0] = vd.b[1] = vd.b[2] = 0.;
    vd.r_lo = lo[0];
    vd.r_step_inv = n[0] > 1 ? (n[0] - 1) / (hi[0] - lo[0]) : 0.;
    vd.phi_lo = lo[1];
    vd.phi_step_inv = n[1] / (2.0 * constant::pi);
    vd.z_lo = lo[2];
    vd.z_step_inv = n[2] > 1 ? (n[2] - 1) / (hi[2] - lo[2]) : 0.;
    vd.nodes = f->nodes;
    *out = f;
    return DPROP_OK;
}

dprop_status dprop_field_destroy(dprop_field* f) {
    if (!f) {
        return DPROP_OK;
    }
    cudaFree(f->nodes);
    delete f;
    return DPROP_OK;
}

dprop_status dprop_propagate(const dprop_config* cfg, const dprop_launch* lc,
                             const dprop_detector* det, const dprop_field* field,
                             const dprop_tracks* tracks,
                             const dprop_results* results, uint64_t n,
                             void* stream) {
    dprop_status s = check_config(cfg);
    if (s != DPROP_OK) {
        return s;
    }
    if (!det || !field || !tracks || !results) {
        return fail(DPROP_E_INVALID, "propagate: NULL argument");
    }
    if (n == 0) {
        return DPROP_OK;
    }
    for (int i = 0; i < 3; ++i) {
        if (!tracks->pos[i] || !tracks->dir[i]) {
            return fail(DPROP_E_INVALID, "propagate: missing track array");
        }
    }
    if (!tracks->time || !tracks->qop || !results->status) {
        return fail(DPROP_E_INVALID, "propagate: missing track/status array");
    }
    if (lc && lc->precision == 8u) {
        return dprop::api::propagate_fp64(*cfg, lc, det, field, *tracks,
                                          *results, n,
                                          static_cast<cudaStream_t>(stream));
    }
    if (lc && lc->precision != 0u && lc->precision != 4u) {
        return fail(DPROP_E_INVALID, "propagate: precision must be 0, 4 or 8");
    }
    const io_ptrs<float> io = make_io<float>(*tracks, *results);
    return launch<float>(*cfg, lc, det, field, io, n,
                         static_cast<cudaStream_t>(stream));
}

dprop_status dprop_propagate_host(const dprop_config* cfg,
                                  const dprop_launch* lc,
                                  const dprop_detector* det,
                                  const dprop_field* field,
                                  const dprop_tracks* tracks,
                                  const dprop_results* results, uint64_t n) {
    dprop_status s = check_config(cfg);
    if (s != DPROP_OK) {
        return s;
    }
    if (!det || !field || !tracks || !results || !results->status) {
        return fail(DPROP_E_INVALID, "propagate_host: NULL argument");
    }
    if (n == 0) {
        if (results->rec_offsets) {
            results->rec_offsets[0] = 0u;
        }
        return DPROP_OK;
    }
    if (results->rec_offsets) {
        return propagate_host_jagged(*cfg, lc, det, field, *tracks, *results, n);
    }
    const uint64_t cap = cfg->max_records;
    // device scratch: inputs (8 doubles), per-track outputs, records
    const size_t in_bytes = 8 * n * sizeof(double);
    const size_t trk_bytes = n * (1 + 6 * 4 + 4 + 8 * 4) + 16 * 256;
    const size_t rec_bytes = cap * n * (8 + 6 * 4 + 21 * 4 + 4 + 1);
    s = ensure_scratch(in_bytes + trk_bytes + rec_bytes + 4096);
    if (s != DPROP_OK) {
        return s;
    }
    char* p = static_cast<char*>(g_scratch.buf);
    auto take = [&](size_t bytes) {
        char* r = p;
        p += (bytes + 255) & ~size_t(255);
        return r;
    };
    const double* d_trk[8];
    for (int i = 0; i < 8; ++i) {
        d_trk[i] = reinterpret_cast<const double*>(take(n * sizeof(double)));
    }
    const void* h_trk[8] = {tracks->pos[0], tracks->pos[1], tracks->pos[2],
                            tracks->time,   tracks->dir[0], tracks->dir[1],
                            tracks->dir[2], tracks->qop};
    for (int i = 0; i < 8; ++i) {
        if (!h_trk[i]) {
            return fail(DPROP_E_INVALID, "propagate_host: missing track array");
        }
        DPROP_CUDA(cudaMemcpyAsync(const_cast<double*>(d_trk[i]), h_trk[i],
                                   n * sizeof(double), cudaMemcpyHostToDevice, 0));
    }
    dprop_results dr{};
    dr.status = reinterpret_cast<uint8_t*>(take(n));
    dr.n_records = results->n_records ? reinterpret_cast<uint32_t*>(take(4 * n)) : nullptr;
    dr.n_steps = results->n_steps ? reinterpret_cast<uint32_t*>(take(4 * n)) : nullptr;
    dr.n_trials = results->n_trials ? reinterpret_cast<uint32_t*>(take(4 * n)) : nullptr;
    dr.path_length = results->path_length ? take(4 * n) : nullptr;
    for (int i = 0; i < 8; ++i) {
        dr.final_free[i] = results->final_free[i] ? take(4 * n) : nullptr;
    }
    dr.rec_barcode = results->rec_barcode ? reinterpret_cast<uint64_t*>(take(8 * cap * n)) : nullptr;
    for (int i = 0; i < 6; ++i) {
        dr.rec_bound[i] = results->rec_bound[i] ? take(4 * cap * n) : nullptr;
    }
    for (int i = 0; i < 21; ++i) {
        dr.rec_cov[i] = results->rec_cov[i] ? take(4 * cap * n) : nullptr;
    }
    dr.rec_path = results->rec_path ? take(4 * cap * n) : nullptr;
    dr.rec_flags = results->rec_flags ? reinterpret_cast<uint8_t*>(take(cap * n)) : nullptr;
    dr.n_intersections = results->n_intersections ? reinterpret_cast<uint32_t*>(take(4 * n)) : nullptr;
    dr.n_transports = results->n_transports ? reinterpret_cast<uint32_t*>(take(4 * n)) : nullptr;
    dr.n_material = results->n_material ? reinterpret_cast<uint32_t*>(take(4 * n)) : nullptr;

    dprop_tracks dt{};
    for (int i = 0; i < 3; ++i) {
        dt.pos[i] = d_trk[i];
        dt.dir[i] = d_trk[4 + i];
    }
    dt.time = d_trk[3];
    dt.qop = d_trk[7];
    const io_ptrs<double> io = make_io<double>(dt, dr);
    s = launch<double>(*cfg, lc, det, field, io, n, 0);
    if (s != DPROP_OK) {
        return s;
    }
    auto d2h = [&](void* h, const void* d, size_t bytes) -> dprop_status {
        if (h && d) {
            DPROP_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, 0));
        }
        return DPROP_OK;
    };
    if ((s = d2h(results->status, dr.status, n)) != DPROP_OK) return s;
    if ((s = d2h(results->n_records, dr.n_records, 4 * n)) != DPROP_OK) return s;
    if ((s = d2h(results->n_steps, dr.n_steps, 4 * n)) != DPROP_OK) return s;
    if ((s = d2h(results->n_trials, dr.n_trials, 4 * n)) != DPROP_OK) return s;
    if ((s = d2h(results->path_length, dr.path_length, 4 * n)) != DPROP_OK) return s;
    for (int i = 0; i < 8; ++i) {
        if ((s = d2h(results->final_free[i], dr.final_free[i], 4 * n)) != DPROP_OK) return s;
    }
    if ((s = d2h(results->rec_barcode, dr.rec_barcode, 8 * cap * n)) != DPROP_OK) return s;
    for (int i = 0; i < 6; ++i) {
        if ((s = d2h(results->rec_bound[i], dr.rec_bound[i], 4 * cap * n)) != DPROP_OK) return s;
    }
    for (int i = 0; i < 21; ++i) {
        if ((s = d2h(results->rec_cov[i], dr.rec_cov[i], 4 * cap * n)) != DPROP_OK) return s;
    }
    if ((s = d2h(results->rec_path, dr.rec_path, 4 * cap * n)) != DPROP_OK) return s;
    if ((s = d2h(results->rec_flags, dr.rec_flags, cap * n)) != DPROP_OK) return s;
    if ((s = d2h(results->n_intersections, dr.n_intersections, 4 * n)) != DPROP_OK) return s;
    if ((s = d2h(results->n_transports, dr.n_transports, 4 * n)) != DPROP_OK) return s;
    if ((s = d2h(results->n_material, dr.n_material, 4 * n)) != DPROP_OK) return s;
    DPROP_CUDA(cudaStreamSynchronize(0));
    return DPROP_OK;
}

dprop_status dprop_release_cache(void) {
    std::lock_guard<std::mutex> lock(g_graph_mutex);
    DPROP_CUDA(cudaDeviceSynchronize());
    for (graph_entry& e : g_graphs) {
        destroy_entry(e);
    }
    g_graphs.clear();
    cudaFree(g_sort.buf);
    g_sort = sort_scratch{};
    cudaFree(g_rounds.buf);
    g_rounds = sort_scratch{};
    cudaFree(g_scratch.buf);
    g_scratch.buf = nullptr;
    g_scratch.bytes = 0;
    for (int k = 0; k < k_pipe_slots; ++k) {
        cudaFree(g_pipe[k].dev);
        g_pipe[k].dev = nullptr;
        g_pipe[k].dev_bytes = 0;
    }
    dprop::api::release_fp64_scratch();
    return DPROP_OK;
}

}  // extern "C"

// ===================================================== allocation-free path
// dprop_propagate_noalloc: the direction-sorted plain propagation with its
// sort scratch in a fixed device array instead of library allocations.
namespace {

// Layout of the fixed scratch: four track-index-sized arrays (sort keys and
// indices, the two halves of each double buffer) followed by the radix-sort
// temporary storage (digit histograms and look-back state only).
constexpr size_t k_noalloc_array_bytes =
    static_cast<size_t>(DPROP_NOALLOC_MAX_TRACKS) * sizeof(uint32_t);
constexpr size_t k_noalloc_temp_offset = 4 * k_noalloc_array_bytes;
constexpr size_t k_noalloc_temp_bytes =
    static_cast<size_t>(DPROP_NOALLOC_SCRATCH_BYTES) - k_noalloc_temp_offset;
static_assert(k_noalloc_temp_offset < DPROP_NOALLOC_SCRATCH_BYTES,
              "no-alloc scratch too small for the sort arrays");

// The scratch itself.  In host code this name is only a stand-in for the
// symbol: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char
    g_noalloc_scratch[DPROP_NOALLOC_SCRATCH_BYTES];

constexpr int k_noalloc_max_devices = 64;
void* g_noalloc_device_ptr[k_noalloc_max_devices] = {};
std::mutex g_noalloc_mutex;

// Device address of the scratch on the current device.  Outside a stream
// capture it is looked up on every call (cheap once the module is loaded),
// so that an address that changed - the module is loaded again after a
// cudaDeviceReset - is picked up; inside a capture (where the lookup, which
// may load the module, must not run) the address of the last call on this
// device is used, so the first call on a device must come before any
// capture.
dprop_status noalloc_scratch(cudaStream_t stream, void** out) {
    int dev = 0;
    DPROP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= k_noalloc_max_devices) {
        return fail(DPROP_E_INVALID, "propagate_noalloc: device index out of range");
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    DPROP_CUDA(cudaStreamIsCapturing(stream, &cap));
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
        }
        g_noalloc_device_ptr[dev] = p;
    } else if (g_noalloc_device_ptr[dev] == nullptr) {
        return fail(DPROP_E_INVALID,
                    "propagate_noalloc: the first call on a device must not "
                    "be inside a stream capture");
    }
    *out = g_noalloc_device_ptr[dev];
    return DPROP_OK;
}

}  // namespace

extern "C" dprop_status dprop_propagate_noalloc(const dprop_config* cfg,
                                                const dprop_detector* det,
                                                const dprop_field* field,
                                                const dprop_tracks* tracks,
                                                const dprop_results* results,
                                                uint64_t n, void* stream_ptr) {
    dprop_status s = check_config(cfg);
    if (s != DPROP_OK) {
        return s;
    }
    if (!det || !field || !tracks || !results) {
        return fail(DPROP_E_INVALID, "propagate_noalloc: NULL argument");
    }
    if (n > DPROP_NOALLOC_MAX_TRACKS) {
        return fail(DPROP_E_INVALID,
                    "propagate_noalloc: " + std::to_string(n) +
                        " tracks exceed the fixed scratch capacity of " +
                        std::to_string(DPROP_NOALLOC_MAX_TRACKS) +
                        " tracks per call; split the batch");
    }
    if (n == 0) {
        return DPROP_OK;
    }
    for (int i = 0; i < 3; ++i) {
        if (!tracks->pos[i] || !tracks->dir[i]) {
            return fail(DPROP_E_INVALID, "propagate_noalloc: missing track array");
        }
    }
    if (!tracks->time || !tracks->qop || !results->status) {
        return fail(DPROP_E_INVALID,
                    "propagate_noalloc: missing track/status array");
    }
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    void* scratch = nullptr;
    s = noalloc_scratch(stream, &scratch);
    if (s != DPROP_OK) {
        return s;
    }
    const int ni = static_cast<int>(n);
    char* base = static_cast<char*>(scratch);
    // keys and indices ping-pong between the in and out arrays (the radix
    // sort's double-buffer form), so its temporary storage holds only the
    // digit histograms and look-back state, not another copy of each array
    cub::DoubleBuffer<uint32_t> keys(
        reinterpret_cast<uint32_t*>(base),
        reinterpret_cast<uint32_t*>(base + k_noalloc_array_bytes));
    cub::DoubleBuffer<uint32_t> order(
        reinterpret_cast<uint32_t*>(base + 2 * k_noalloc_array_bytes),
        reinterpret_cast<uint32_t*>(base + 3 * k_noalloc_array_bytes));
    size_t temp_bytes = 0;
    DPROP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys,
                                               order, ni, 0, 20, stream));
    if (temp_bytes > k_noalloc_temp_bytes) {
        return fail(DPROP_E_INVALID,
                    "propagate_noalloc: radix-sort storage exceeds the fixed "
                    "scratch");
    }
    void* temp = base + k_noalloc_temp_offset;

    const io_ptrs<float> io = make_io<float>(*tracks, *results);
    const unsigned int key_grid = static_cast<unsigned int>((n + 255) / 256);
    direction_key_kernel<float><<<key_grid, 256, 0, stream>>>(
        io.trk[4], io.trk[5], io.trk[6], io.trk[7], n, keys.Current(),
        order.Current());
    DPROP_CUDA(cudaGetLastError());
    DPROP_CUDA(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, order,
                                               ni, 0, 20, stream));
    const prop_cfg<float> pc = make_prop_cfg<float>(*cfg);
    launch_plain_mb<float, DPROP_MIN_BLOCKS>(k_plain_block, stream, det,
                                             field->view, pc, io, n,
                                             order.Current());
    DPROP_CUDA(cudaGetLastError());
    return DPROP_OK;
}
