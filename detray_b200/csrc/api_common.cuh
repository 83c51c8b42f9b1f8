// Pieces of the C ABI implementation shared by its translation units
// (dprop_api.cu: propagation; adjoint_api.cu: adjoint mode and the reverse
// sweep): error reporting, the detector and field handles, the direction
// sort of the inputs and the register-budget choice of a launch.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "core/propagate.cuh"
#include "detray_b200/dprop.h"

namespace dprop::api {

// Record msg as dprop_last_error() of this thread and return s.
dprop_status fail(dprop_status s, const std::string& msg);
dprop_status cuda_fail(cudaError_t e, const char* what);

// Register budget of a launch: resident CTAs of 128 threads per SM, one of
// 8 (64 registers), 12 (40) or 16 (32).
int occupancy_of(const dprop_launch* lc);

// Device scratch bytes of enqueue_direction_sort for n tracks.
size_t sort_scratch_bytes(uint64_t n);

// Enqueue the sort of n tracks by direction, charge and pT (20-bit key,
// CUB radix sort) on stream; *order receives the device array of sorted track
// indices, which lives in scratch.  No allocation, no synchronisation.
dprop_status enqueue_direction_sort(const float* dx, const float* dy,
                                    const float* dz, const float* dq,
                                    uint64_t n, void* scratch,
                                    size_t scratch_bytes, cudaStream_t stream,
                                    const uint32_t** order);
dprop_status enqueue_direction_sort(const double* dx, const double* dy,
                                    const double* dz, const double* dq,
                                    uint64_t n, void* scratch,
                                    size_t scratch_bytes, cudaStream_t stream,
                                    const uint32_t** order);

}  // namespace dprop::api

#define DPROP_CUDA(call)                                      \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) {                              \
            return ::dprop::api::cuda_fail(e_, #call);        \
        }                                                     \
    } while (0)

struct dprop_detector {
    int device{0};
    dprop::dev_volume* volumes{nullptr};
    dprop::dev_surface* surfaces{nullptr};
    dprop::dev_mask<float>* masks{nullptr};
    dprop::dev_transform<float>* transforms{nullptr};
    dprop::dev_slab<float>* slabs{nullptr};
    uint32_t* bf_surfaces{nullptr};
    dprop::dev_grid<float>* grids{nullptr};
    uint32_t* grid_bins{nullptr};
    uint32_t* vol_material{nullptr};  // NULL: no volume carries material
    // double-precision copies of the floating-point tables (fp64 launches)
    dprop::dev_mask<double>* masks_d{nullptr};
    dprop::dev_transform<double>* transforms_d{nullptr};
    dprop::dev_slab<double>* slabs_d{nullptr};
    dprop::dev_grid<double>* grids_d{nullptr};
    uint32_t n_volumes{0}, n_surfaces{0};
    // the detector holds line surfaces, material rods, multi-entry grid bins,
    // material maps or volume material: launches use the kernels that
    // include the code for them
    bool wires{false};
    dprop::detector_view<double> view_d() const { return view_d_as<true>(); }
    template <bool W>
    dprop::detector_view<double, W> view_d_as() const {
        dprop::detector_view<double, W> v;
        v.volumes = volumes;
        v.surfaces = surfaces;
        v.masks = masks_d;
        v.transforms = transforms_d;
        v.slabs = slabs_d;
        v.bf_surfaces = bf_surfaces;
        v.grids = grids_d;
        v.grid_bins = grid_bins;
        v.vol_material = vol_material;
        v.n_volumes = n_volumes;
        v.n_surfaces = n_surfaces;
        return v;
    }
    dprop::detector_view<float> view() const { return view_as<true>(); }
    template <bool W>
    dprop::detector_view<float, W> view_as() const {
        dprop::detector_view<float, W> v;
        v.volumes = volumes;
        v.surfaces = surfaces;
        v.masks = masks;
        v.transforms = transforms;
        v.slabs = slabs;
        v.bf_surfaces = bf_surfaces;
        v.grids = grids;
        v.grid_bins = grid_bins;
        v.vol_material = vol_material;
        v.n_volumes = n_volumes;
        v.n_surfaces = n_surfaces;
        return v;
    }
};

struct dprop_field {
    int device{0};
    float4* nodes{nullptr};
    dprop::field_view<float> view{};
    dprop::field_view<double> view_d{};  // same nodes, double arithmetic
};

namespace dprop::api {

// fp64 propagation (dprop_launch.precision == 8): double inputs, arithmetic
// and results; plain one-thread-per-track kernel, optional direction sort.
dprop_status propagate_fp64(const dprop_config& cfg, const dprop_launch* lc,
                            const dprop_detector* det, const dprop_field* field,
                            const dprop_tracks& tracks,
                            const dprop_results& results, uint64_t n,
                            cudaStream_t stream);

// Frees the grow-only scratch of fp64 launches (dprop_release_cache).
void release_fp64_scratch();

}  // namespace dprop::api
