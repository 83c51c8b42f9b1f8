// Round-based propagation (dprop_launch.method = DPROP_METHOD_PERSISTENT).
//
// The plain form runs the whole propagation loop of a track in one thread:
// the lanes of a warp diverge at every surface, every navigation
// re-initialisation and every track end, and the full state of the loop
// (about 500 bytes a track) has to live in registers and the thread's stack
// across all of it.  Here the loop is cut into the segments of
// core/machine.cuh and each track's state lives in device memory between
// them (core/slots.cuh, one array per field, indexed by the track's slot in
// the direction-sorted batch).  Every round:
//
//   queue_count_kernel / queue_scatter_kernel
//       read the one-byte next-segment array of all slots and write the
//       slots of each phase, in slot (= direction) order, into the work
//       queues of the step and navigation phases;
//   rounds_fast_kernel
//       the step phase: RK steps with the high-trust navigation update,
//       the path-limit aborter and the surface actors (transport, material,
//       setter, recorder), until a track needs the volume-level navigation
//       update or ends.  A warp stops its round once fewer than yield_lanes
//       of its lanes can still step (a warp vote after every step), so that
//       warps do not run on with a few lanes;
//   rounds_nav_kernel
//       the navigation update's cache re-evaluation, volume switch and local
//       navigation (grid and portal search), with all lanes of a warp doing
//       it at once.
//
// Every sort_interval rounds (dprop_launch.sort_interval, 0: never) both
// queues are re-sorted by volume before the phases run (queue_key_kernel +
// a stable 8-bit radix sort): the step phase by the volume a track is in,
// the navigation phase by the volume it enters, so that the lanes of a warp
// intersect the same kinds of surfaces and walk the same grids and portal
// lists.  Inside a volume the slot (direction) order stays.
//
// Each phase kernel is persistent: a grid of the SMs' resident CTAs whose
// warps pull 32 queue entries at a time from a device counter until the
// queue is empty.  Once fewer than tail_tracks tracks are alive (the count
// kernel decides it on the device), that round's step phase runs them to
// their end with every segment inline, as rounds_tail_kernel does after
// the last round.  Records are staged as one 128-byte (fp32) or 256-byte
// (fp64) row per record and converted to the result layout at the end
// (rounds_unstage_kernel).  Each kernel loads and stores only the state its
// segments use; the segments perform the loop's operations in its order,
// so a track driven through the phases ends as it would in the one-shot
// loop (bit for bit in a host build of both; on the device the separately
// compiled kernels may contract multiply-adds differently in the last
// bits).  Everything is templated on the arithmetic type: fp32, and fp64
// for dprop_launch.precision = 8.
#include <cuda_runtime.h>

#include <cub/block/block_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#include <type_traits>

#include "api_common.cuh"
#include "core/phases.cuh"
#include "track_io.cuh"

using namespace dprop;

namespace {

constexpr int k_build_threads = 256;  // 16 slots each: one tile per CTA
static_assert(k_build_threads * 16 == static_cast<int>(k_queue_tile),
              "queue tile = 16 slots per thread");
constexpr int k_phase_block = 128;
constexpr uint32_t k_unstage_ways = 8u;

// Queue of a segment: 0 step phase, 2 navigation, -1 ended (queue 1 holds
// tracks waiting for the surface actors, which the step phase runs itself,
// so it stays empty).  merged: every live slot in queue 0 (the tail).
__device__ __forceinline__ int queue_of(uint32_t pc, bool merged) {
    if (pc == pc_done) {
        return -1;
    }
    if (merged) {
        return 0;
    }
    if (pc == pc_surf) {
        return 1;
    }
    if (pc == pc_nav) {
        return 2;
    }
    return 0;
}

// Work-queue state of one propagation: three queues of slot indices, their
// lengths, the per-tile counts of the builder and the pull counters of the
// phase kernels.
struct queue_set {
    uint32_t* q[3];
    uint32_t* count;   // [4]: queue lengths, [3] = 1 when the round runs the
                       // remaining tracks to their end (merged)
    uint32_t* pull;    // [3]
    uint32_t* ticket;  // CTAs of the count kernel done
    uint32_t* tiles;   // [3 * n_tiles]: counts, then the tiles' offsets
};

__device__ __forceinline__ void unpack16(uint4 v, uint32_t* b) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    for (int i = 0; i < 4; ++i) {
        for (int j = 0; j < 4; ++j) {
            b[4 * i + j] = (w[i] >> (8 * j)) & 0xffu;
        }
    }
}

// Sort key of each queue entry: the volume the track's next phase works in
// (for a track on a portal in the navigation queue, the volume the portal
// leads to), 0xff past the queue's end.
template <typename S>
__global__ void __launch_bounds__(k_build_threads)
    queue_key_kernel(const uint32_t* __restrict__ q,
                     const uint32_t* __restrict__ count,
                     const __grid_constant__ slot_soa<S> s,
                     uint8_t* __restrict__ keys, uint64_t n, int nav_queue) {
    const uint32_t cnt = *count;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         i < n; i += stride) {
        if (i >= cnt) {
            keys[i] = 0xffu;
            continue;
        }
        const uint64_t slot = q[i];
        uint32_t vol = s.volume[slot];
        if (nav_queue) {
            const uint32_t nb = s.nav_bytes[slot];
            const int next = static_cast<int>(nb & 0xffu);
            const int8_t status = static_cast<int8_t>((nb >> 16) & 0xffu);
            if (status == e_on_portal && next >= 1 && next <= k_cache + 1) {
                candidate<S> c;
                load_cand(s, slot, next - 1, c);
                if (c.volume_link != static_cast<uint16_t>(k_invalid_link)) {
                    vol = c.volume_link;
                }
            }
        }
        keys[i] = static_cast<uint8_t>(vol % 255u);
    }
}

// Block-wide exclusive sum of three counters per thread; returns the totals.
__device__ void block_scan3(const uint32_t (&v)[3], uint32_t (&excl)[3],
                            uint32_t (&total)[3]) {
    using scan_t = cub::BlockScan<uint32_t, k_build_threads>;
    __shared__ typename scan_t::TempStorage tmp;
    for (int k = 0; k < 3; ++k) {
        scan_t(tmp).ExclusiveSum(v[k], excl[k], total[k]);
        __syncthreads();
    }
}

// Per-tile counts of the slots of each queue.  The CTA that finishes last
// (a ticket taken after a memory fence; no CTA waits for another) turns the
// counts into the tiles' offsets, in place, and sets the queue lengths:
// when fewer than tail_tracks tracks are alive (or merged is set: the last
// round) every live track goes to queue 0 and the round runs them to their
// end.
__global__ void __launch_bounds__(k_build_threads)
    queue_count_kernel(const uint8_t* __restrict__ pc, queue_set qs,
                       uint32_t n_tiles, int merged, uint32_t tail_tracks) {
    if (qs.count[3] != 0u) {
        // the previous round ran every live track to its end: nothing is
        // left, the queues stay empty (count[3] stays set)
        if (blockIdx.x == 0 && threadIdx.x < 3) {
            qs.count[threadIdx.x] = 0u;
        }
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x < 3) {
        qs.pull[threadIdx.x] = 0u;
    }
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * k_queue_tile +
                          static_cast<uint64_t>(threadIdx.x) * 16u;
    uint32_t b[16];
    unpack16(*reinterpret_cast<const uint4*>(pc + base), b);
    uint32_t c[3] = {0u, 0u, 0u};
    for (int i = 0; i < 16; ++i) {
        const int q = queue_of(b[i], false);
        if (q >= 0) {
            ++c[q];
        }
    }
    __shared__ uint32_t part[k_build_threads / 32][3];
    for (int k = 0; k < 3; ++k) {
        uint32_t v = c[k];
        for (int o = 16; o > 0; o >>= 1) {
            v += __shfl_down_sync(0xffffffffu, v, o);
        }
        if ((threadIdx.x & 31u) == 0u) {
            part[threadIdx.x >> 5][k] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        uint32_t v = 0u;
        for (int w = 0; w < k_build_threads / 32; ++w) {
            v += part[w][threadIdx.x];
        }
        qs.tiles[3u * blockIdx.x + threadIdx.x] = v;
    }
    // the last CTA to finish scans the tile counts
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        last = atomicAdd(qs.ticket, 1u) == n_tiles - 1u;
    }
    __syncthreads();
    if (!last) {
        return;
    }
    __threadfence();
    const uint32_t per = (n_tiles + k_build_threads - 1u) / k_build_threads;
    const uint32_t lo = threadIdx.x * per;
    const uint32_t hi = lo + per < n_tiles ? lo + per : n_tiles;
    uint32_t sum[3] = {0u, 0u, 0u};
    for (uint32_t j = lo; j < hi; ++j) {
        for (int k = 0; k < 3; ++k) {
            sum[k] += __ldcg(qs.tiles + 3u * j + k);
        }
    }
    uint32_t excl[3], total[3];
    block_scan3(sum, excl, total);
    const uint32_t live = total[0] + total[1] + total[2];
    const bool m = merged != 0 || live < tail_tracks;
    // in place: each thread rewrites only its own tiles
    uint32_t run[3] = {excl[0], excl[1], excl[2]};
    uint32_t run_m = excl[0] + excl[1] + excl[2];
    for (uint32_t j = lo; j < hi; ++j) {
        uint32_t t[3];
        for (int k = 0; k < 3; ++k) {
            t[k] = __ldcg(qs.tiles + 3u * j + k);
        }
        if (m) {
            qs.tiles[3u * j] = run_m;
            qs.tiles[3u * j + 1] = 0u;
            qs.tiles[3u * j + 2] = 0u;
            run_m += t[0] + t[1] + t[2];
        } else {
            for (int k = 0; k < 3; ++k) {
                qs.tiles[3u * j + k] = run[k];
                run[k] += t[k];
            }
        }
    }
    if (threadIdx.x == 0) {
        qs.count[0] = m ? live : total[0];
        qs.count[1] = m ? 0u : total[1];
        qs.count[2] = m ? 0u : total[2];
        qs.count[3] = m ? 1u : 0u;
        *qs.ticket = 0u;
    }
}

// Slots of each queue in slot order: the tile's offset comes from the count
// kernel, positions inside the tile from a block scan of the per-thread
// counts (three 21-bit fields of one 64-bit value).
__global__ void __launch_bounds__(k_build_threads)
    queue_scatter_kernel(const uint8_t* __restrict__ pc, queue_set qs) {
    const uint32_t tile = blockIdx.x;
    const bool m = qs.count[3] != 0u;
    if (m && qs.count[0] == 0u) {
        return;  // nothing alive
    }
    uint32_t offset[3];
    for (int k = 0; k < 3; ++k) {
        offset[k] = qs.tiles[3u * tile + k];
    }
    const uint64_t base = static_cast<uint64_t>(tile) * k_queue_tile +
                          static_cast<uint64_t>(threadIdx.x) * 16u;
    uint32_t b[16];
    unpack16(*reinterpret_cast<const uint4*>(pc + base), b);
    uint64_t mine = 0u;
    for (int i = 0; i < 16; ++i) {
        const int q = queue_of(b[i], m);
        if (q >= 0) {
            mine += uint64_t(1) << (21 * q);
        }
    }
    using scan_t = cub::BlockScan<uint64_t, k_build_threads>;
    __shared__ typename scan_t::TempStorage scan_tmp;
    uint64_t excl = 0u, total = 0u;
    scan_t(scan_tmp).ExclusiveSum(mine, excl, total);
    uint32_t pos[3];
    for (int k = 0; k < 3; ++k) {
        pos[k] = offset[k] + static_cast<uint32_t>((excl >> (21 * k)) & 0x1fffffu);
    }
    for (int i = 0; i < 16; ++i) {
        const int q = queue_of(b[i], m);
        if (q >= 0) {
            qs.q[q][pos[q]++] = static_cast<uint32_t>(base + i);
        }
    }
}

template <typename S, typename In>
__device__ __forceinline__ record_sink<S> make_sink(
    const api::io_ptrs<In, S>& io, uint64_t n, const prop_cfg<S>& cfg,
    uint32_t* stage) {
    record_sink<S> rec;
    rec.barcode = io.rec_barcode;
    rec.bound = io.rec_bound;
    rec.cov = io.rec_cov;
    rec.path = io.rec_path;
    rec.flags = io.rec_flags;
    rec.n_tracks = n;
    rec.track = 0u;
    rec.capacity = (io.rec_barcode != nullptr) ? cfg.max_records : 0u;
    rec.count = 0u;
    rec.stage = stage;
    return rec;
}

template <typename S, typename In>
__device__ __forceinline__ void write_outputs(const api::io_ptrs<In, S>& io,
                                              uint64_t t,
                                              const track_outputs<S>& o) {
    if (io.status) io.status[t] = o.status;
    if (io.n_records) io.n_records[t] = o.n_records;
    if (io.n_steps) io.n_steps[t] = o.n_steps;
    if (io.n_trials) io.n_trials[t] = o.n_trials;
    if (io.n_isect) io.n_isect[t] = o.n_isect;
    if (io.n_transport) io.n_transport[t] = o.n_transport;
    if (io.n_material) io.n_material[t] = o.n_material;
    if (io.path_length) io.path_length[t] = o.path_length;
    for (int i = 0; i < 8; ++i) {
        if (io.final_free[i]) io.final_free[i][t] = o.fin[i];
    }
}

// Whether the calling warp can find work in a queue of cnt entries: the
// warps pull 32 entries at a time, so warps beyond the number of 32-entry
// chunks leave at once instead of each taking a turn on the pull counter
// (the other warps still take every chunk).
__device__ __forceinline__ bool warp_has_work(uint32_t cnt) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    return warp < (cnt + 31u) / 32u;
}

// Next 32 queue entries for the calling warp (all lanes call it together).
__device__ __forceinline__ uint32_t pull32(uint32_t* pull) {
    uint32_t base = 0u;
    if ((threadIdx.x & 31u) == 0u) {
        base = atomicAdd(pull, 32u);
    }
    return __shfl_sync(0xffffffffu, base, 0);
}

// Propagation start of every slot; pads the next-segment array to whole
// tiles with ended slots.  inv (with staged records) receives the slot of
// each input track.
template <typename S, typename In, bool W>
__global__ void __launch_bounds__(k_phase_block)
    rounds_init_kernel(const __grid_constant__ detector_view<S, W> det,
                       const __grid_constant__ prop_cfg<S> cfg,
                       const __grid_constant__ api::io_ptrs<In, S> io,
                       const __grid_constant__ slot_soa<S> s, uint64_t n,
                       uint64_t n_pad, const uint32_t* __restrict__ order,
                       uint32_t* __restrict__ inv) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t slot = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         slot < n_pad; slot += stride) {
        if (slot >= n) {
            s.pc[slot] = pc_done;
            continue;
        }
        const uint64_t t = order ? static_cast<uint64_t>(order[slot]) : slot;
        if (inv) {
            inv[t] = static_cast<uint32_t>(slot);
        }
        const vec3<S> pos{static_cast<S>(io.trk[0][t]),
                              static_cast<S>(io.trk[1][t]),
                              static_cast<S>(io.trk[2][t])};
        const vec3<S> dir{static_cast<S>(io.trk[4][t]),
                              static_cast<S>(io.trk[5][t]),
                              static_cast<S>(io.trk[6][t])};
        phase_init<S, W>(s, slot, static_cast<uint32_t>(t), pos,
                             static_cast<S>(io.trk[3][t]), dir,
                             static_cast<S>(io.trk[7][t]), det, cfg);
    }
}

// The step phase, compiled for MinBlocks resident CTAs per SM: 3 (up to 168
// registers: the state and the step's temporaries fit without spills), 4
// (128) or 5 (102).  The best budget depends on the workload (more warps
// hide the field map's gather latency), so it is a launch choice.
template <typename S, typename In, bool W, int MinBlocks>
__global__ void __launch_bounds__(k_phase_block, MinBlocks)
    rounds_fast_kernel(const __grid_constant__ detector_view<S, W> det,
                       const __grid_constant__ field_view<S> field,
                       const __grid_constant__ prop_cfg<S> cfg,
                       const __grid_constant__ api::io_ptrs<In, S> io,
                       const __grid_constant__ slot_soa<S> s,
                       const uint32_t* __restrict__ queue,
                       const uint32_t* __restrict__ count, uint32_t* pull,
                       uint64_t n, uint32_t step_budget, uint32_t yield_lanes,
                       uint32_t* stage) {
    const uint32_t cnt = *count;
    if (!warp_has_work(cnt)) {
        return;
    }
    const unsigned lane = threadIdx.x & 31u;
    record_sink<S> rec = make_sink(io, n, cfg, stage);
    if (count[3] != 0u) {
        // few tracks left: run each to its end in this round (the queue
        // builder merged all live tracks into this queue)
        while (true) {
            const uint32_t base = pull32(pull);
            if (base >= cnt) {
                break;
            }
            const uint32_t idx = base + lane;
            if (idx < cnt) {
                const uint64_t slot = queue[idx];
                const track_outputs<S> o =
                    phase_tail<S, W>(s, slot, det, field, cfg, rec);
                write_outputs(io, s.track[slot], o);
            }
            __syncwarp();
        }
        return;
    }
    while (true) {
        const uint32_t base = pull32(pull);
        if (base >= cnt) {
            break;
        }
        const uint32_t idx = base + lane;
        const bool valid = idx < cnt;
        const uint64_t slot = valid ? queue[idx] : 0u;
        nav_cache<S> cache;
        track_state<S> ts;
        bind_cache(ts.nav, cache);
        loop_state<S> ls;
        cand_window win;
        if (valid) {
            fast_load<S, W>(s, slot, ts, ls, win);
        }
        const int n_valid = __popc(__ballot_sync(0xffffffffu, valid));
        bool active = valid;
        for (uint32_t it = 0;; ++it) {
            if (active) {
                const uint8_t pc = fast_advance<S, W>(
                    ts, ls, win, s, slot, det, field, cfg, rec);
                active = machine_is_fast(pc);
            }
            const int m = __popc(__ballot_sync(0xffffffffu, active));
            if (m == 0 || it + 1u >= step_budget ||
                (m < static_cast<int>(yield_lanes) && m < n_valid)) {
                break;
            }
        }
        if (valid) {
            fast_store<S, W>(s, slot, ts, ls, win);
            if (ls.pc == pc_done) {
                write_outputs(io, s.track[slot],
                              fast_outputs(s, slot, ts, ls));
            }
        }
    }
}

// The navigation update's volume-level part.  fp32: 8 resident CTAs per SM
// (64 registers, a few bytes of spills): more warps hide the dependent
// loads of the candidate search (measured on B200 against 4 CTAs, 89
// registers: 24.6 against 25.1 ms on 1 M toy tracks, 118.4 against 120.6
// ms on 4 M tracks in the field map); fp64: 4.
template <typename S, bool W>
__global__ void __launch_bounds__(k_phase_block, sizeof(S) == 4 ? 8 : 4)
    rounds_nav_kernel(const __grid_constant__ detector_view<S, W> det,
                      const __grid_constant__ prop_cfg<S> cfg,
                      const __grid_constant__ slot_soa<S> s,
                      const uint32_t* __restrict__ queue,
                      const uint32_t* __restrict__ count, uint32_t* pull) {
    const uint32_t cnt = *count;
    if (!warp_has_work(cnt)) {
        return;
    }
    while (true) {
        const uint32_t base = pull32(pull);
        if (base >= cnt) {
            break;
        }
        const uint32_t idx = base + (threadIdx.x & 31u);
        if (idx < cnt) {
            phase_nav<S, W>(s, queue[idx], det, cfg);
        }
        __syncwarp();
    }
}

// The tracks still alive after the last round, every segment inline.
template <typename S, typename In, bool W>
__global__ void __launch_bounds__(k_phase_block, 8)
    rounds_tail_kernel(const __grid_constant__ detector_view<S, W> det,
                       const __grid_constant__ field_view<S> field,
                       const __grid_constant__ prop_cfg<S> cfg,
                       const __grid_constant__ api::io_ptrs<In, S> io,
                       const __grid_constant__ slot_soa<S> s,
                       const uint32_t* __restrict__ queue,
                       const uint32_t* __restrict__ count, uint32_t* pull,
                       uint64_t n, uint32_t* stage) {
    const uint32_t cnt = *count;
    record_sink<S> rec = make_sink(io, n, cfg, stage);
    while (true) {
        const uint32_t base = pull32(pull);
        if (base >= cnt) {
            break;
        }
        const uint32_t idx = base + (threadIdx.x & 31u);
        if (idx < cnt) {
            const uint64_t slot = queue[idx];
            const track_outputs<S> o =
                phase_tail<S, W>(s, slot, det, field, cfg, rec);
            write_outputs(io, s.track[slot], o);
        }
        __syncwarp();
    }
}

// Staged records to the public slot-major arrays: thread (t, y) converts
// records y, y + k_unstage_ways, ... of input track t, so that most
// records are in flight at once and consecutive threads write consecutive
// words of every array.
template <typename S, typename In>
__global__ void __launch_bounds__(k_phase_block)
    rounds_unstage_kernel(const __grid_constant__ prop_cfg<S> cfg,
                          const __grid_constant__ api::io_ptrs<In, S> io,
                          const uint32_t* __restrict__ rec_count,
                          const uint32_t* __restrict__ inv,
                          const uint32_t* __restrict__ stage, uint64_t n) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) {
        return;
    }
    const record_sink<S> out = make_sink(io, n, cfg, nullptr);
    const uint64_t slot = inv[t];
    const uint32_t c = rec_count[slot];
    const uint32_t m = c < out.capacity ? c : out.capacity;
    for (uint32_t k = blockIdx.y; k < m; k += gridDim.y) {
        unstage_record<S>(stage, slot, k, t, out);
    }
}

// Resident CTAs of a kernel on the current device (the persistent grid).
template <typename K>
dprop_status resident_grid(K kernel, unsigned int* grid) {
    int dev = 0, sms = 0, per_sm = 0;
    DPROP_CUDA(cudaGetDevice(&dev));
    DPROP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    DPROP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, kernel, k_phase_block, 0));
    per_sm = per_sm < 1 ? 1 : per_sm;
    *grid = static_cast<unsigned int>(sms * per_sm);
    return DPROP_OK;
}

template <typename S>
struct rounds_layout {
    slot_soa<S> slots;
    queue_set qs;
    uint64_t n_tiles;
    uint8_t* keys[2];        // volume re-sort: keys in, keys out
    uint32_t* nav_sorted;    // the navigation queue re-sorted (the step
                             // queue goes to the unused queue 1)
    void* sort_temp;
    size_t sort_temp_bytes;
    uint32_t* inv;    // slot of each input track (staged records only)
    uint32_t* stage;  // staged records, rec_cap per slot (or null)
};

size_t al256(size_t b) { return (b + 255u) & ~size_t(255u); }

// Scratch layout: slot arrays, three queues, counters and tile counts, and
// with rec_cap > 0 the record staging area and the input -> slot map.
template <typename S>
size_t rounds_layout_bytes(uint64_t n, bool wires, uint32_t rec_cap,
                           rounds_layout<S>* out, void* base) {
    const uint64_t n_tiles = queue_tiles(n);
    slot_soa<S> s{};
    const size_t slot_bytes = carve_slots<S>(base, n, wires, &s);
    size_t off = al256(slot_bytes);
    char* p = static_cast<char*>(base);
    queue_set qs{};
    for (int k = 0; k < 3; ++k) {
        qs.q[k] = reinterpret_cast<uint32_t*>(p + off);
        off += al256(n * 4u);
    }
    qs.count = reinterpret_cast<uint32_t*>(p + off);
    qs.pull = qs.count + 4;
    qs.ticket = qs.count + 8;
    off += 256;
    qs.tiles = reinterpret_cast<uint32_t*>(p + off);
    off += al256(3u * n_tiles * 4u);
    uint8_t* keys[2];
    for (int k = 0; k < 2; ++k) {
        keys[k] = reinterpret_cast<uint8_t*>(p + off);
        off += al256(n);
    }
    uint32_t* nav_sorted = reinterpret_cast<uint32_t*>(p + off);
    off += al256(n * 4u);
    size_t temp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(
        nullptr, temp_bytes, static_cast<const uint8_t*>(nullptr),
        static_cast<uint8_t*>(nullptr), static_cast<const uint32_t*>(nullptr),
        static_cast<uint32_t*>(nullptr), static_cast<int>(n), 0, 8);
    void* sort_temp = p + off;
    off += al256(temp_bytes);
    uint32_t* inv = nullptr;
    uint32_t* stage = nullptr;
    if (rec_cap > 0u) {
        inv = reinterpret_cast<uint32_t*>(p + off);
        off += al256(n * 4u);
        stage = reinterpret_cast<uint32_t*>(p + off);
        off += al256(n * rec_cap * (4u * staged_record_words<S>()));
    }
    if (out) {
        out->slots = s;
        out->qs = qs;
        out->n_tiles = n_tiles;
        out->inv = inv;
        out->stage = stage;
        out->keys[0] = keys[0];
        out->keys[1] = keys[1];
        out->nav_sorted = nav_sorted;
        out->sort_temp = sort_temp;
        out->sort_temp_bytes = temp_bytes;
    }
    return off;
}

template <typename S, typename In, bool W, int FastBlocks>
dprop_status enqueue_rounds_w(const detector_view<S, W>& det,
                              const field_view<S>& field,
                              const prop_cfg<S>& cfg,
                              const api::io_ptrs<In, S>& io, uint64_t n,
                              const uint32_t* order, const rounds_layout<S>& L,
                              uint32_t rounds, uint32_t step_budget,
                              uint32_t yield_lanes, uint32_t sort_interval,
                              uint32_t tail_tracks, cudaStream_t st,
                              cudaEvent_t mark, uint32_t mark_round) {
    const uint64_t n_pad = L.n_tiles * k_queue_tile;
    const unsigned int tiles = static_cast<unsigned int>(L.n_tiles);
    unsigned int g_init = 0, g_fast = 0, g_nav = 0, g_tail = 0;
    dprop_status s = DPROP_OK;
    if ((s = resident_grid(rounds_init_kernel<S, In, W>, &g_init)) != DPROP_OK ||
        (s = resident_grid(rounds_fast_kernel<S, In, W, FastBlocks>, &g_fast)) != DPROP_OK ||
        (s = resident_grid(rounds_nav_kernel<S, W>, &g_nav)) != DPROP_OK ||
        (s = resident_grid(rounds_tail_kernel<S, In, W>, &g_tail)) != DPROP_OK) {
        return s;
    }
    DPROP_CUDA(cudaMemsetAsync(L.qs.ticket, 0, sizeof(uint32_t), st));
    // count[3] (the last round ran the tail) from an earlier call
    DPROP_CUDA(cudaMemsetAsync(L.qs.count, 0, 4 * sizeof(uint32_t), st));
    rounds_init_kernel<S, In, W><<<g_init, k_phase_block, 0, st>>>(
        det, cfg, io, L.slots, n, n_pad, order, L.inv);
    DPROP_CUDA(cudaGetLastError());
    for (uint32_t r = 0; r <= rounds; ++r) {
        const int merged = (r == rounds) ? 1 : 0;
        queue_count_kernel<<<tiles, k_build_threads, 0, st>>>(
            L.slots.pc, L.qs, tiles, merged, tail_tracks);
        queue_scatter_kernel<<<tiles, k_build_threads, 0, st>>>(L.slots.pc,
                                                                L.qs);
        DPROP_CUDA(cudaGetLastError());
        if (merged) {
            rounds_tail_kernel<S, In, W><<<g_tail, k_phase_block, 0, st>>>(
                det, field, cfg, io, L.slots, L.qs.q[0], L.qs.count,
                L.qs.pull, n, L.stage);
            DPROP_CUDA(cudaGetLastError());
            if (L.stage != nullptr) {
                // 8 record indices in flight per track (a track has ~8
                // records); more mostly launches threads that find no record
                // after two dependent loads
                const dim3 ug(static_cast<unsigned int>(
                                  (n + k_phase_block - 1) / k_phase_block),
                              cfg.max_records < k_unstage_ways
                                  ? cfg.max_records : k_unstage_ways);
                rounds_unstage_kernel<S, In><<<ug, k_phase_block, 0, st>>>(
                    cfg, io, L.slots.rec_count, L.inv, L.stage, n);
                DPROP_CUDA(cudaGetLastError());
            }
            break;
        }
        const uint32_t* q_fast = L.qs.q[0];
        const uint32_t* q_nav = L.qs.q[2];
        if (sort_interval > 0u && r > 0u && r % sort_interval == 0u) {
            const unsigned int kg = static_cast<unsigned int>(
                (n + k_build_threads - 1) / k_build_threads);
            for (int k = 0; k < 2; ++k) {
                const int qi = 2 * k;  // step queue 0, navigation queue 2
                uint32_t* dst = k == 0 ? L.qs.q[1] : L.nav_sorted;
                queue_key_kernel<S><<<kg, k_build_threads, 0, st>>>(
                    L.qs.q[qi], L.qs.count + qi, L.slots, L.keys[0], n, k);
                DPROP_CUDA(cudaGetLastError());
                size_t tb = L.sort_temp_bytes;
                DPROP_CUDA(cub::DeviceRadixSort::SortPairs(
                    L.sort_temp, tb, L.keys[0], L.keys[1], L.qs.q[qi], dst,
                    static_cast<int>(n), 0, 8, st));
            }
            q_fast = L.qs.q[1];
            q_nav = L.nav_sorted;
        }
        rounds_fast_kernel<S, In, W, FastBlocks><<<g_fast, k_phase_block, 0, st>>>(
            det, field, cfg, io, L.slots, q_fast, L.qs.count, L.qs.pull, n,
            step_budget, yield_lanes, L.stage);
        rounds_nav_kernel<S, W><<<g_nav, k_phase_block, 0, st>>>(
            det, cfg, L.slots, q_nav, L.qs.count + 2, L.qs.pull + 2);
        DPROP_CUDA(cudaGetLastError());
        if (mark && r == mark_round) {
            DPROP_CUDA(cudaEventRecord(mark, st));
        }
    }
    if (mark && mark_round >= rounds) {
        DPROP_CUDA(cudaEventRecord(mark, st));
    }
    return DPROP_OK;
}

}  // namespace

namespace dprop::api {

constexpr uint32_t k_default_steps_per_round = 16u;
constexpr uint32_t k_default_rounds = 64u;
constexpr uint32_t k_default_yield_lanes = 16u;
// default tail threshold: n / 64 live tracks
constexpr uint64_t k_default_tail_div = 64u;

size_t rounds_scratch_bytes(uint64_t n, bool wires, uint32_t rec_cap) {
    return rounds_layout_bytes<float>(n, wires, rec_cap, nullptr, nullptr) +
           256u;
}

size_t rounds_scratch_bytes_fp64(uint64_t n, bool wires, uint32_t rec_cap) {
    return rounds_layout_bytes<double>(n, wires, rec_cap, nullptr, nullptr) +
           256u;
}

namespace {

// The detector and field views in the arithmetic type S.
template <typename S, bool W>
detector_view<S, W> det_view(const dprop_detector* det) {
    if constexpr (sizeof(S) == 8) {
        return det->view_d_as<W>();
    } else {
        return det->view_as<W>();
    }
}

template <typename S>
const field_view<S>& fld_view(const dprop_field* field) {
    if constexpr (sizeof(S) == 8) {
        return field->view_d;
    } else {
        return field->view;
    }
}

// The round-based propagation in S; the step phase's register budgets the
// kernels are built for: fp32 3, 4 or 5 resident CTAs per SM (default 4),
// fp64 2 or 3 (default 2: twice the registers for the same state).
template <typename S, typename In>
dprop_status enqueue_rounds_s(const dprop_launch* lc, const dprop_detector* det,
                              const dprop_field* field,
                              const prop_cfg<S>& cfg,
                              const io_ptrs<In, S>& io, uint64_t n,
                              const uint32_t* order, void* scratch,
                              size_t scratch_bytes, cudaStream_t stream,
                              cudaEvent_t mark, uint32_t mark_round) {
    constexpr bool fp64 = sizeof(S) == 8;
    if (n > 0x7fffffffull) {
        return fail(DPROP_E_INVALID, "persistent method: n_tracks too large");
    }
    if (cfg.step.field_gradient) {
        return fail(DPROP_E_UNSUPPORTED,
                    "persistent method: use_field_gradient runs with the "
                    "plain method only");
    }
    const uint32_t rec_cap = staged_capacity(cfg, io);
    const size_t need = fp64 ? rounds_scratch_bytes_fp64(n, det->wires, rec_cap)
                             : rounds_scratch_bytes(n, det->wires, rec_cap);
    if (scratch_bytes < need) {
        return fail(DPROP_E_INVALID, "persistent method: scratch too small");
    }
    void* base = reinterpret_cast<void*>(
        (reinterpret_cast<uintptr_t>(scratch) + 255u) & ~uintptr_t(255u));
    rounds_layout<S> L{};
    rounds_layout_bytes<S>(n, det->wires, rec_cap, &L, base);
    const uint32_t rounds = (lc && lc->rounds) ? lc->rounds : k_default_rounds;
    const uint32_t budget = (lc && lc->steps_per_round) ? lc->steps_per_round
                                                        : k_default_steps_per_round;
    const uint32_t yield = (lc && lc->yield_lanes) ? lc->yield_lanes
                                                   : k_default_yield_lanes;
    const uint32_t sort_interval = lc ? lc->sort_interval : 0u;
    // live tracks below which a round runs the rest to their end
    const uint32_t tail_tracks =
        (lc && lc->tail_tracks) ? lc->tail_tracks
                                : static_cast<uint32_t>(n / k_default_tail_div);
    if (rounds > 100000u || yield > 32u) {
        return fail(DPROP_E_INVALID,
                    "persistent method: rounds > 100000 or yield_lanes > 32");
    }
    if (lc && lc->block_size != 0u && lc->block_size != k_phase_block) {
        return fail(DPROP_E_INVALID,
                    "persistent method: block_size must be 0 or 128");
    }
    const uint32_t fb =
        (lc && lc->ctas_per_sm) ? lc->ctas_per_sm : (fp64 ? 2u : 4u);
    if (fp64 ? (fb < 2u || fb > 3u) : (fb < 3u || fb > 5u)) {
        return fail(DPROP_E_INVALID,
                    fp64 ? "persistent method, fp64: ctas_per_sm must be 0, "
                           "2 or 3"
                         : "persistent method: ctas_per_sm must be 0, 3, 4 "
                           "or 5");
    }
    auto go = [&](auto fast_blocks) -> dprop_status {
        constexpr int FB = decltype(fast_blocks)::value;
        if (det->wires) {
            return enqueue_rounds_w<S, In, true, FB>(
                det_view<S, true>(det), fld_view<S>(field), cfg, io, n, order,
                L, rounds, budget, yield, sort_interval, tail_tracks, stream,
                mark, mark_round);
        }
        return enqueue_rounds_w<S, In, false, FB>(
            det_view<S, false>(det), fld_view<S>(field), cfg, io, n, order, L,
            rounds, budget, yield, sort_interval, tail_tracks, stream, mark,
            mark_round);
    };
    if constexpr (fp64) {
        if (fb == 3u) {
            return go(std::integral_constant<int, 3>{});
        }
        return go(std::integral_constant<int, 2>{});
    } else {
        if (fb == 3u) {
            return go(std::integral_constant<int, 3>{});
        }
        if (fb == 5u) {
            return go(std::integral_constant<int, 5>{});
        }
        return go(std::integral_constant<int, 4>{});
    }
}

}  // namespace

template <typename In>
dprop_status enqueue_rounds(const dprop_launch* lc, const dprop_detector* det,
                            const dprop_field* field,
                            const prop_cfg<float>& cfg, const io_ptrs<In>& io,
                            uint64_t n, const uint32_t* order, void* scratch,
                            size_t scratch_bytes, cudaStream_t stream,
                            cudaEvent_t mark, uint32_t mark_round) {
    return enqueue_rounds_s<float, In>(lc, det, field, cfg, io, n, order,
                                       scratch, scratch_bytes, stream, mark,
                                       mark_round);
}

dprop_status enqueue_rounds_fp64(const dprop_launch* lc,
                                 const dprop_detector* det,
                                 const dprop_field* field,
                                 const prop_cfg<double>& cfg,
                                 const io_ptrs<double, double>& io,
                                 uint64_t n, const uint32_t* order,
                                 void* scratch, size_t scratch_bytes,
                                 cudaStream_t stream) {
    return enqueue_rounds_s<double, double>(lc, det, field, cfg, io, n, order,
                                            scratch, scratch_bytes, stream,
                                            nullptr, 0u);
}

template dprop_status enqueue_rounds<float>(const dprop_launch*,
                                            const dprop_detector*,
                                            const dprop_field*,
                                            const prop_cfg<float>&,
                                            const io_ptrs<float>&, uint64_t,
                                            const uint32_t*, void*, size_t,
                                            cudaStream_t, cudaEvent_t,
                                            uint32_t);
template dprop_status enqueue_rounds<double>(const dprop_launch*,
                                             const dprop_detector*,
                                             const dprop_field*,
                                             const prop_cfg<float>&,
                                             const io_ptrs<double>&, uint64_t,
                                             const uint32_t*, void*, size_t,
                                             cudaStream_t, cudaEvent_t,
                                             uint32_t);

}  // namespace dprop::api
