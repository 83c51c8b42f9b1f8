// Helix truth scan for navigation validation: the C ABI entry points
// dprop_helix_scan and dprop_validate_navigation (dprop.h).
//
// Kernels:
//   helix_scan_kernel    one thread per (track, surface) pair: the track's
//                        helix intersected with one surface (core/helix.cuh);
//                        hits inside a mask and along the track are appended
//                        to the track's slots with an atomic counter
//   scan_finish_kernel   one thread per track: sort the hits by |path|
//                        (ties by surface index, which is the reference's
//                        stable order over the surface list) and cut after
//                        the first hit that leaves the world
//   validate_kernel      one thread per track: holes and extra surfaces of
//                        a propagation's records against the scan
// The surfaces of a detector are read by every track: they stay in L2.
#include <cuda_runtime.h>

#include "api_common.cuh"
#include "core/helix.cuh"

using namespace dprop;
using dprop::api::fail;

namespace {

constexpr int k_scan_block = 128;

template <typename S>
struct scan_io {
    const S* trk[8];
    uint8_t* status;
    uint32_t* n_hits;
    uint64_t* barcode;
    S* path;
    S* loc[2];
    uint16_t* volume_link;
    uint32_t capacity;
};

template <typename S, bool W>
__global__ void __launch_bounds__(k_scan_block)
    helix_scan_kernel(const __grid_constant__ detector_view<S, W> det,
                      const __grid_constant__ scan_io<S> io, vec3<S> bfield,
                      S mask_tol, uint64_t n) {
    const uint64_t t = blockIdx.x;
    const uint32_t sf_idx = blockIdx.y * k_scan_block + threadIdx.x;
    if (t >= n || sf_idx >= det.n_surfaces) {
        return;
    }
    helix<S> h;
    h.init(vec3<S>{io.trk[0][t], io.trk[1][t], io.trk[2][t]},
           vec3<S>{io.trk[4][t], io.trk[5][t], io.trk[6][t]}, io.trk[7][t],
           bfield);
    const root_cfg<S> cfg{S(unit::um), 1000u, S(5000) * S(unit::mm)};
    const uint32_t cap = io.capacity;
    helix_surface_hits(det, sf_idx, h, mask_tol, cfg,
                       [&](const scan_hit<S>& hit) {
                           const uint32_t k = atomicAdd(io.n_hits + t, 1u);
                           if (k < cap) {
                               const uint64_t o =
                                   static_cast<uint64_t>(k) * n + t;
                               io.barcode[o] = det.surfaces[hit.sf].barcode;
                               io.path[o] = hit.path;
                               if (io.loc[0]) io.loc[0][o] = hit.loc0;
                               if (io.loc[1]) io.loc[1][o] = hit.loc1;
                               io.volume_link[o] = hit.volume_link;
                           }
                       });
}

template <typename S>
__device__ void swap_hits(const scan_io<S>& io, uint64_t a, uint64_t b) {
    const uint64_t bc = io.barcode[a];
    io.barcode[a] = io.barcode[b];
    io.barcode[b] = bc;
    const S p = io.path[a];
    io.path[a] = io.path[b];
    io.path[b] = p;
    for (int i = 0; i < 2; ++i) {
        if (io.loc[i]) {
            const S l = io.loc[i][a];
            io.loc[i][a] = io.loc[i][b];
            io.loc[i][b] = l;
        }
    }
    const uint16_t v = io.volume_link[a];
    io.volume_link[a] = io.volume_link[b];
    io.volume_link[b] = v;
}

// surface index of a barcode (bits 27..47)
__device__ __forceinline__ uint64_t sf_key(uint64_t bc) {
    return (bc >> 27) & 0x1fffffu;
}

template <typename S>
__global__ void __launch_bounds__(k_scan_block)
    scan_finish_kernel(const __grid_constant__ scan_io<S> io, uint64_t n) {
    const uint64_t t =
        static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) {
        return;
    }
    const uint32_t found = io.n_hits[t];
    if (found == 0u) {
        io.status[t] = DPROP_SCAN_EMPTY;
        return;
    }
    if (found > io.capacity) {
        io.status[t] = DPROP_SCAN_OVERFLOW;
        return;
    }
    // insertion sort of the track's slots by (|path|, surface index)
    for (uint32_t i = 1; i < found; ++i) {
        for (uint32_t j = i; j > 0; --j) {
            const uint64_t a = static_cast<uint64_t>(j - 1) * n + t;
            const uint64_t b = static_cast<uint64_t>(j) * n + t;
            const S pa = fabs(io.path[a]);
            const S pb = fabs(io.path[b]);
            const bool after = pa > pb || (pa == pb && sf_key(io.barcode[a]) >
                                                          sf_key(io.barcode[b]));
            if (!after) {
                break;
            }
            swap_hits(io, a, b);
        }
    }
    uint32_t kept = found;
    for (uint32_t k = 0; k < found; ++k) {
        if (io.volume_link[static_cast<uint64_t>(k) * n + t] ==
            static_cast<uint16_t>(DPROP_INVALID_LINK)) {
            kept = k + 1u;
            break;
        }
    }
    io.n_hits[t] = kept;
    io.status[t] = DPROP_SCAN_OK;
}

template <typename S>
dprop_status launch_scan(const dprop_detector* det, const double b[3],
                         const dprop_tracks* tracks, uint64_t n,
                         double mask_tol, const dprop_scan_results* r,
                         cudaStream_t st) {
    scan_io<S> io{};
    for (int i = 0; i < 3; ++i) {
        io.trk[i] = static_cast<const S*>(tracks->pos[i]);
        io.trk[4 + i] = static_cast<const S*>(tracks->dir[i]);
    }
    io.trk[3] = static_cast<const S*>(tracks->time);
    io.trk[7] = static_cast<const S*>(tracks->qop);
    io.status = r->status;
    io.n_hits = r->n_hits;
    io.barcode = r->barcode;
    io.path = static_cast<S*>(r->path);
    io.loc[0] = static_cast<S*>(r->loc[0]);
    io.loc[1] = static_cast<S*>(r->loc[1]);
    io.volume_link = r->volume_link;
    io.capacity = r->capacity;
    const vec3<S> bf{static_cast<S>(b[0]), static_cast<S>(b[1]),
                     static_cast<S>(b[2])};
    DPROP_CUDA(cudaMemsetAsync(r->n_hits, 0, n * sizeof(uint32_t), st));
    const unsigned int sf_blocks =
        (det->n_surfaces + k_scan_block - 1) / k_scan_block;
    if (sf_blocks > 0u) {
        const dim3 grid(static_cast<unsigned int>(n), sf_blocks);
        if constexpr (sizeof(S) == 8) {
            if (det->wires) {
                helix_scan_kernel<S, true><<<grid, k_scan_block, 0, st>>>(
                    det->view_d(), io, bf, static_cast<S>(mask_tol), n);
            } else {
                detector_view<S, false> v;
                const detector_view<S, true> w = det->view_d();
                v.volumes = w.volumes;
                v.surfaces = w.surfaces;
                v.masks = w.masks;
                v.transforms = w.transforms;
                v.slabs = w.slabs;
                v.bf_surfaces = w.bf_surfaces;
                v.grids = w.grids;
                v.grid_bins = w.grid_bins;
                v.n_volumes = w.n_volumes;
                v.n_surfaces = w.n_surfaces;
                helix_scan_kernel<S, false><<<grid, k_scan_block, 0, st>>>(
                    v, io, bf, static_cast<S>(mask_tol), n);
            }
        } else {
            if (det->wires) {
                helix_scan_kernel<S, true><<<grid, k_scan_block, 0, st>>>(
                    det->view_as<true>(), io, bf, static_cast<S>(mask_tol), n);
            } else {
                helix_scan_kernel<S, false><<<grid, k_scan_block, 0, st>>>(
                    det->view_as<false>(), io, bf, static_cast<S>(mask_tol),
                    n);
            }
        }
        DPROP_CUDA(cudaGetLastError());
    }
    const unsigned int tb =
        static_cast<unsigned int>((n + k_scan_block - 1) / k_scan_block);
    scan_finish_kernel<S><<<tb, k_scan_block, 0, st>>>(io, n);
    DPROP_CUDA(cudaGetLastError());
    return DPROP_OK;
}

template <typename Ti, typename Tr>
__global__ void __launch_bounds__(k_scan_block)
    validate_kernel(const uint8_t* __restrict__ scan_status,
                    const uint32_t* __restrict__ n_hits,
                    const uint64_t* __restrict__ truth_bc,
                    const Ti* __restrict__ truth_path,
                    const uint16_t* __restrict__ truth_vlink,
                    const uint8_t* __restrict__ rec_status,
                    const uint32_t* __restrict__ n_records,
                    const uint64_t* __restrict__ rec_bc,
                    const Tr* __restrict__ rec_path, uint32_t max_records,
                    uint64_t n, double path_tol, uint32_t* n_missed,
                    uint32_t* n_extra) {
    const uint64_t t =
        static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) {
        return;
    }
    const uint32_t nt = (scan_status[t] == DPROP_SCAN_OK) ? n_hits[t] : 0u;
    const uint32_t nr = n_records[t] < max_records ? n_records[t] : max_records;
    uint32_t missed, extra;
    compare_trace(truth_bc, truth_path, truth_vlink, nt, rec_bc, rec_path, nr,
                  rec_status[t] == DPROP_TRK_EXITED, n, t, path_tol, missed,
                  extra);
    n_missed[t] = missed;
    n_extra[t] = extra;
}

template <typename Ti, typename Tr>
void launch_validate(const dprop_scan_results* s, const dprop_results* r,
                     uint32_t max_records, uint64_t n, double tol,
                     const dprop_validation* out, cudaStream_t st) {
    const unsigned int tb =
        static_cast<unsigned int>((n + k_scan_block - 1) / k_scan_block);
    validate_kernel<Ti, Tr><<<tb, k_scan_block, 0, st>>>(
        s->status, s->n_hits, s->barcode, static_cast<const Ti*>(s->path),
        s->volume_link, r->status, r->n_records, r->rec_barcode,
        static_cast<const Tr*>(r->rec_path), max_records, n, tol,
        out->n_missed, out->n_extra);
}

}  // namespace

extern "C" {

dprop_status dprop_validate_navigation(const dprop_scan_results* s,
                                       const dprop_results* r,
                                       uint32_t record_precision,
                                       uint32_t max_records, uint64_t n,
                                       double path_tolerance,
                                       const dprop_validation* out,
                                       void* stream) {
    if (!s || !r || !out) {
        return fail(DPROP_E_INVALID, "validate_navigation: NULL argument");
    }
    if ((s->precision != 4u && s->precision != 8u) ||
        (record_precision != 4u && record_precision != 8u)) {
        return fail(DPROP_E_INVALID,
                    "validate_navigation: precision must be 4 or 8");
    }
    if (!(path_tolerance >= 0.0)) {
        return fail(DPROP_E_INVALID,
                    "validate_navigation: negative path tolerance");
    }
    if (n == 0) {
        return DPROP_OK;
    }
    if (n > 0x7fffffffull) {
        return fail(DPROP_E_INVALID, "validate_navigation: too many tracks");
    }
    if (!s->status || !s->n_hits || !s->barcode || !s->path ||
        !s->volume_link || !r->status || !r->n_records ||
        (max_records > 0u && (!r->rec_barcode || !r->rec_path)) ||
        !out->n_missed || !out->n_extra) {
        return fail(DPROP_E_INVALID, "validate_navigation: missing array");
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (s->precision == 8u) {
        if (record_precision == 8u) {
            launch_validate<double, double>(s, r, max_records, n,
                                            path_tolerance, out, st);
        } else {
            launch_validate<double, float>(s, r, max_records, n,
                                           path_tolerance, out, st);
        }
    } else {
        if (record_precision == 8u) {
            launch_validate<float, double>(s, r, max_records, n,
                                           path_tolerance, out, st);
        } else {
            launch_validate<float, float>(s, r, max_records, n,
                                          path_tolerance, out, st);
        }
    }
    DPROP_CUDA(cudaGetLastError());
    return DPROP_OK;
}

dprop_status dprop_helix_scan(const dprop_detector* det, const double b[3],
                              const dprop_tracks* tracks, uint64_t n,
                              double mask_tolerance,
                              const dprop_scan_results* r, void* stream) {
    if (!det || !b || !tracks || !r) {
        return fail(DPROP_E_INVALID, "helix_scan: NULL argument");
    }
    if (r->precision != 4u && r->precision != 8u) {
        return fail(DPROP_E_INVALID, "helix_scan: precision must be 4 or 8");
    }
    const double bb = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
    if (!(bb > 0.0) || !(bb < 1e30)) {
        return fail(DPROP_E_INVALID,
                    "helix_scan: the field must be finite and non-zero");
    }
    if (!(mask_tolerance >= 0.0) || !(mask_tolerance < 1e3)) {
        return fail(DPROP_E_INVALID,
                    "helix_scan: mask_tolerance must be in [0, 1000) mm");
    }
    if (n == 0) {
        return DPROP_OK;
    }
    if (n > 0x7fffffffull) {
        return fail(DPROP_E_INVALID, "helix_scan: too many tracks");
    }
    for (int i = 0; i < 3; ++i) {
        if (!tracks->pos[i] || !tracks->dir[i]) {
            return fail(DPROP_E_INVALID, "helix_scan: missing track array");
        }
    }
    if (!tracks->time || !tracks->qop || !r->status || !r->n_hits ||
        !r->volume_link || (r->capacity > 0u && (!r->barcode || !r->path))) {
        return fail(DPROP_E_INVALID, "helix_scan: missing array");
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (r->precision == 8u) {
        return launch_scan<double>(det, b, tracks, n, mask_tolerance, r, st);
    }
    return launch_scan<float>(det, b, tracks, n, mask_tolerance, r, st);
}

}  // extern "C"
