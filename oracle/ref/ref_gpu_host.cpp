/*
 * REFERENCE GPU BASELINE — measurement infrastructure only.
 *
 * Host driver of the reference's own CUDA propagation kernel (ref_gpu.cu),
 * compiled from the reference's headers where they lie in the reference
 * checkout.  vecmem (not vendored) is replaced by the stand-in under
 * oracle/shim, whose view types carry device annotations
 * under nvcc; the toy detector is built by the reference's own builder into
 * CUDA managed memory, so that its host views are valid in device code (as
 * in the reference benchmark's managed-memory variant); covfie's constant
 * field is replaced by a constant field with the same at(x, y, z).
 *
 * Exported: refgpu_toy_bench() (constant field, the benchmark kernel) and
 * refgpu_toy_map_bench() (field map, the tutorial's kernel with the path-limit
 * aborter).  Built by oracle/ref/Makefile into
 * oracle/_ref/libdetray_ref_gpu.so; only bench.py's reference GPU row calls
 * it.
 */
#include <cuda_runtime.h>

#include <cassert>

#include "detray/test/common/build_toy_detector.hpp"
#include "detray_b200/dprop.h"
#include "ref_gpu.hpp"

#include <limits>
#include <new>
#include <string>
#include <vector>

using namespace refgpu;

namespace {

thread_local std::string g_error;

// CUDA managed memory behind the detector's and the tracks' containers
struct managed_resource final : public vecmem::memory_resource {
    void* do_allocate(std::size_t bytes, std::size_t) override {
        void* p = nullptr;
        if (cudaMallocManaged(&p, bytes > 0 ? bytes : 1) != cudaSuccess) {
            throw std::bad_alloc();
        }
        return p;
    }
    void do_deallocate(void* p, std::size_t, std::size_t) override {
        cudaFree(p);
    }
    bool do_is_equal(const std::pmr::memory_resource& o) const noexcept override {
        return this == &o;
    }
};

propagation::config to_ref_config(const dprop_config& c) {
    propagation::config p{};
    p.stepping.min_stepsize = c.min_stepsize;
    p.stepping.rk_error_tol = c.rk_error_tol;
    p.stepping.step_constraint = c.step_constraint;
    p.stepping.path_limit = c.path_limit;
    p.stepping.max_rk_updates = c.max_rk_updates;
    p.stepping.use_mean_loss = c.use_mean_loss != 0;
    p.stepping.use_eloss_gradient = c.use_eloss_gradient != 0;
    p.stepping.use_field_gradient = c.use_field_gradient != 0;
    p.stepping.do_covariance_transport = c.do_covariance_transport != 0;
    p.navigation.intersection.min_mask_tolerance = c.min_mask_tolerance;
    p.navigation.intersection.max_mask_tolerance = c.max_mask_tolerance;
    p.navigation.intersection.mask_tolerance_scalor = c.mask_tolerance_scalor;
    p.navigation.intersection.path_tolerance = c.path_tolerance;
    p.navigation.intersection.overstep_tolerance = c.overstep_tolerance;
    p.navigation.search_window = {c.search_window[0], c.search_window[1]};
    p.navigation.accumulated_error = c.accumulated_error;
    p.navigation.n_scattering_stddev = c.n_scattering_stddev;
    p.navigation.estimate_scattering_noise = c.estimate_scattering_noise != 0;
    return p;
}

#define REF_CUDA(call)                                                    \
    do {                                                                  \
        const cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) {                                          \
            g_error = std::string(#call) + ": " + cudaGetErrorString(e_); \
            return 2;                                                     \
        }                                                                 \
    } while (0)

}  // namespace

extern "C" {

const char* refgpu_last_error(void) { return g_error.c_str(); }

/// Time the reference's CUDA propagation of n tracks (rows x, y, z, t, tx,
/// ty, tz, q/p as doubles) through the toy detector (4 barrel layers, 7
/// end-cap discs per side, 0.15 mm modules) in a constant field bz along z:
/// warmup untimed launches, then steps launches timed with CUDA events.
/// ms_per_step gets the mean launch time, n_exited the number of tracks whose
/// propagate() returned true in the last launch.
int refgpu_toy_bench(const dprop_config* c, double bz,
                     const double* const* trk, uint64_t n, int warmup,
                     int steps, double* ms_per_step, uint64_t* n_exited) {
    try {
        if (n == 0 || n > 0x7fffffffu) {
            g_error = "refgpu_toy_bench: n out of range";
            return 1;
        }
        managed_resource mr;
        toy_det_config<scalar> tcfg{};
        tcfg.n_brl_layers(4u).n_edc_layers(7u).module_mat_thickness(0.15f);
        auto [det, names] = build_toy_detector<algebra_t>(mr, tcfg);
        vecmem::vector<track_t> tracks(&mr);
        tracks.reserve(n);
        for (uint64_t t = 0; t < n; ++t) {
            track_t p{};
            p.set_pos({static_cast<scalar>(trk[0][t]),
                       static_cast<scalar>(trk[1][t]),
                       static_cast<scalar>(trk[2][t])});
            p.set_time(static_cast<scalar>(trk[3][t]));
            p.set_dir({static_cast<scalar>(trk[4][t]),
                       static_cast<scalar>(trk[5][t]),
                       static_cast<scalar>(trk[6][t])});
            p.set_qop(static_cast<scalar>(trk[7][t]));
            tracks.push_back(p);
        }
        const propagation::config cfg = to_ref_config(*c);
        typename chain_t::state_tuple blueprint{};
        typename chain_t::state_tuple* d_states = nullptr;
        uint8_t* d_status = nullptr;
        REF_CUDA(cudaMalloc(&d_states, sizeof(blueprint)));
        REF_CUDA(cudaMemcpy(d_states, &blueprint, sizeof(blueprint),
                            cudaMemcpyHostToDevice));
        REF_CUDA(cudaMalloc(&d_status, n));
        const const_field field{{0.f, 0.f, static_cast<scalar>(bz)}};
        const auto det_view = det.get_data();
        const vecmem::data::vector_view<track_t> tracks_view(
            static_cast<unsigned int>(n), tracks.data());
        cudaEvent_t e0, e1;
        REF_CUDA(cudaEventCreate(&e0));
        REF_CUDA(cudaEventCreate(&e1));
        const unsigned int nn = static_cast<unsigned int>(n);
        for (int i = 0; i < warmup; ++i) {
            if (launch(cfg, det_view, field, d_states, tracks_view, d_status,
                       nn) != 0) {
                g_error = "reference kernel launch failed";
                return 2;
            }
        }
        REF_CUDA(cudaDeviceSynchronize());
        REF_CUDA(cudaEventRecord(e0));
        for (int i = 0; i < steps; ++i) {
            launch(cfg, det_view, field, d_states, tracks_view, d_status, nn);
        }
        REF_CUDA(cudaEventRecord(e1));
        REF_CUDA(cudaEventSynchronize(e1));
        REF_CUDA(cudaGetLastError());
        float ms = 0.f;
        REF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        *ms_per_step = static_cast<double>(ms) / (steps > 0 ? steps : 1);
        std::vector<uint8_t> status(n);
        REF_CUDA(cudaMemcpy(status.data(), d_status, n, cudaMemcpyDeviceToHost));
        uint64_t ok = 0;
        for (uint8_t s : status) {
            ok += (s != 0u) ? 1u : 0u;
        }
        *n_exited = ok;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(d_states);
        cudaFree(d_status);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

/// Time the reference tutorial's CUDA propagation (path-limit aborter,
/// parameter updater with the material interactor, ref_map_kernel) of n
/// tracks through the toy detector in a field map on an (r, phi, z) node
/// grid: lo/hi/nn as dprop_field_create_grid, values (B_r, B_phi, B_z) per
/// node.  Timing and outputs as refgpu_toy_bench.
int refgpu_toy_map_bench(const dprop_config* c, const double* lo,
                         const double* hi, const uint32_t* nn,
                         const float* values, const double* const* trk,
                         uint64_t n, int warmup, int steps,
                         double* ms_per_step, uint64_t* n_exited) {
    try {
        if (n == 0 || n > 0x7fffffffu) {
            g_error = "refgpu_toy_map_bench: n out of range";
            return 1;
        }
        managed_resource mr;
        toy_det_config<scalar> tcfg{};
        tcfg.n_brl_layers(4u).n_edc_layers(7u).module_mat_thickness(0.15f);
        auto [det, names] = build_toy_detector<algebra_t>(mr, tcfg);
        vecmem::vector<track_t> tracks(&mr);
        tracks.reserve(n);
        for (uint64_t t = 0; t < n; ++t) {
            track_t p{};
            p.set_pos({static_cast<scalar>(trk[0][t]),
                       static_cast<scalar>(trk[1][t]),
                       static_cast<scalar>(trk[2][t])});
            p.set_time(static_cast<scalar>(trk[3][t]));
            p.set_dir({static_cast<scalar>(trk[4][t]),
                       static_cast<scalar>(trk[5][t]),
                       static_cast<scalar>(trk[6][t])});
            p.set_qop(static_cast<scalar>(trk[7][t]));
            tracks.push_back(p);
        }
        const uint64_t n_nodes = static_cast<uint64_t>(nn[0]) * nn[1] * nn[2];
        std::vector<float4> h_nodes(n_nodes);
        for (uint64_t i = 0; i < n_nodes; ++i) {
            h_nodes[i] = make_float4(values[3 * i], values[3 * i + 1],
                                     values[3 * i + 2], 0.f);
        }
        float4* d_nodes = nullptr;
        uint8_t* d_status = nullptr;
        REF_CUDA(cudaMalloc(&d_nodes, n_nodes * sizeof(float4)));
        REF_CUDA(cudaMemcpy(d_nodes, h_nodes.data(), n_nodes * sizeof(float4),
                            cudaMemcpyHostToDevice));
        REF_CUDA(cudaMalloc(&d_status, n));
        map_field field{};
        field.nodes = d_nodes;
        for (int i = 0; i < 3; ++i) {
            field.n[i] = nn[i];
            field.lo[i] = static_cast<scalar>(lo[i]);
        }
        field.step_inv[0] = nn[0] > 1 ? static_cast<scalar>((nn[0] - 1) / (hi[0] - lo[0])) : 0.f;
        field.step_inv[1] = static_cast<scalar>(nn[1] / 6.283185307179586);
        field.step_inv[2] = nn[2] > 1 ? static_cast<scalar>((nn[2] - 1) / (hi[2] - lo[2])) : 0.f;
        const propagation::config cfg = to_ref_config(*c);
        const scalar path_limit = c->use_path_limit_aborter
                                      ? static_cast<scalar>(c->path_limit)
                                      : std::numeric_limits<scalar>::max();
        const auto det_view = det.get_data();
        const vecmem::data::vector_view<track_t> tracks_view(
            static_cast<unsigned int>(n), tracks.data());
        cudaEvent_t e0, e1;
        REF_CUDA(cudaEventCreate(&e0));
        REF_CUDA(cudaEventCreate(&e1));
        const unsigned int m = static_cast<unsigned int>(n);
        for (int i = 0; i < warmup; ++i) {
            if (launch_map(cfg, path_limit, det_view, field, tracks_view,
                           d_status, m) != 0) {
                g_error = "reference map kernel launch failed";
                return 2;
            }
        }
        REF_CUDA(cudaDeviceSynchronize());
        REF_CUDA(cudaEventRecord(e0));
        for (int i = 0; i < steps; ++i) {
            launch_map(cfg, path_limit, det_view, field, tracks_view, d_status,
                       m);
        }
        REF_CUDA(cudaEventRecord(e1));
        REF_CUDA(cudaEventSynchronize(e1));
        REF_CUDA(cudaGetLastError());
        float ms = 0.f;
        REF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        *ms_per_step = static_cast<double>(ms) / (steps > 0 ? steps : 1);
        std::vector<uint8_t> status(n);
        REF_CUDA(cudaMemcpy(status.data(), d_status, n, cudaMemcpyDeviceToHost));
        uint64_t ok = 0;
        for (uint8_t st : status) {
            ok += (st != 0u) ? 1u : 0u;
        }
        *n_exited = ok;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(d_nodes);
        cudaFree(d_status);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

}  // extern "C"
