// Propagation with the direct navigator: the C ABI entry point
// dprop_propagate_direct (dprop.h).
//
// Kernel:
//   propagate_direct_kernel  one thread per track: the propagation loop of
//                            core/propagate.cuh with the direct navigation
//                            policy of core/direct.cuh, starting from free
//                            tracks or from bound parameters on a surface,
//                            walking the track's surface sequence forward or
//                            backward; records as dprop_propagate.
#include <cuda_runtime.h>

#include "api_common.cuh"
#include "core/config.hpp"
#include "core/direct.cuh"
#include "track_io.cuh"

using namespace dprop;
using dprop::api::fail;

namespace {

constexpr int k_direct_block = 128;

struct direct_io {
    const uint64_t* sequence;
    const uint32_t* length;
    uint32_t max_length;
    float direction;
    const uint64_t* start_barcode;
    const float* start_bound[6];
};

template <bool W>
__global__ void __launch_bounds__(k_direct_block)
    propagate_direct_kernel(const __grid_constant__ detector_view<float, W> det,
                            const __grid_constant__ field_view<float> field,
                            const __grid_constant__ prop_cfg<float> cfg,
                            const __grid_constant__ api::io_ptrs<float> io,
                            const __grid_constant__ direct_io dio,
                            uint64_t n) {
    const uint64_t t =
        static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) {
        return;
    }
    vec3<float> pos, dir;
    float time, qop;
    bool start_ok = true;
    if (dio.start_barcode != nullptr) {
        const uint32_t sf = barcode_index(dio.start_barcode[t]);
        float b[6];
        for (int i = 0; i < 6; ++i) {
            b[i] = dio.start_bound[i][t];
        }
        if (sf < det.n_surfaces) {
            bound_start(det, sf, b, pos, dir, time, qop);
        } else {
            start_ok = false;
            pos = {0.f, 0.f, 0.f};
            dir = {0.f, 0.f, 1.f};
            time = 0.f;
            qop = b[4];
        }
    } else {
        pos = {io.trk[0][t], io.trk[1][t], io.trk[2][t]};
        dir = {io.trk[4][t], io.trk[5][t], io.trk[6][t]};
        time = io.trk[3][t];
        qop = io.trk[7][t];
    }

    nav_cache<float> cache;
    track_state<float> ts;
    bind_cache(ts.nav, cache);
    init_track_state(ts, pos, time, dir, qop, cfg);
    ts.nav.direction = dio.direction;

    direct_navigation<float> navigator;
    navigator.sequence = dio.sequence;
    navigator.n_tracks = n;
    navigator.track = t;
    const uint32_t len = dio.length[t];
    navigator.length = static_cast<int32_t>(
        len < dio.max_length ? len : dio.max_length);
    navigator.next_external = 0;
    navigator.reset(ts.nav, det);

    record_sink<float> rec;
    rec.barcode = io.rec_barcode;
    rec.bound = io.rec_bound;
    rec.cov = io.rec_cov;
    rec.path = io.rec_path;
    rec.flags = io.rec_flags;
    rec.n_tracks = n;
    rec.track = t;
    rec.capacity = (io.rec_barcode != nullptr) ? cfg.max_records : 0u;
    rec.stage = nullptr;
    rec.count = 0u;

    uint8_t status = DPROP_TRK_NO_SURFACE;
    if (start_ok) {
        status = propagate_track_with(navigator, ts, det, field, cfg, rec,
                                      no_tape{});
    }

    if (io.status) io.status[t] = status;
    if (io.n_records) io.n_records[t] = rec.count;
    if (io.n_steps) io.n_steps[t] = ts.step.n_steps;
    if (io.n_trials) io.n_trials[t] = ts.step.n_trials;
    if (io.n_isect) io.n_isect[t] = ts.nav.n_isect;
    if (io.n_transport) io.n_transport[t] = ts.n_transport;
    if (io.n_material) io.n_material[t] = ts.n_material;
    if (io.path_length) {
        io.path_length[t] = static_cast<float>(ts.step.path_length);
    }
    const float fin[8] = {ts.step.pos.x, ts.step.pos.y, ts.step.pos.z,
                          ts.step.time,  ts.step.dir.x, ts.step.dir.y,
                          ts.step.dir.z, ts.step.qop};
    for (int i = 0; i < 8; ++i) {
        if (io.final_free[i]) io.final_free[i][t] = fin[i];
    }
}

}  // namespace

extern "C" {

dprop_status dprop_propagate_direct(const dprop_config* cfg,
                                    const dprop_detector* det,
                                    const dprop_field* field,
                                    const dprop_tracks* tracks,
                                    const dprop_sequence* seq,
                                    const dprop_results* results, uint64_t n,
                                    void* stream) {
    if (!cfg || !det || !field || !seq || !results) {
        return fail(DPROP_E_INVALID, "propagate_direct: NULL argument");
    }
    if (cfg->use_field_gradient || cfg->use_eloss_gradient ||
        det->vol_material != nullptr) {
        return fail(DPROP_E_UNSUPPORTED,
                    "propagate_direct: field/eloss gradients and volume "
                    "material are not supported by the direct navigator");
    }
    if (cfg->max_iterations == 0u) {
        return fail(DPROP_E_INVALID,
                    "propagate_direct: max_iterations must be > 0");
    }
    if (seq->direction != 1 && seq->direction != -1) {
        return fail(DPROP_E_INVALID,
                    "propagate_direct: direction must be +1 or -1");
    }
    if (n == 0) {
        return DPROP_OK;
    }
    if (!seq->length || (seq->max_length > 0u && !seq->barcodes)) {
        return fail(DPROP_E_INVALID, "propagate_direct: missing sequence");
    }
    if (seq->start_barcode) {
        for (int i = 0; i < 6; ++i) {
            if (!seq->start_bound[i]) {
                return fail(DPROP_E_INVALID,
                            "propagate_direct: missing start_bound array");
            }
        }
    } else {
        if (!tracks) {
            return fail(DPROP_E_INVALID,
                        "propagate_direct: no tracks and no bound start");
        }
        for (int i = 0; i < 3; ++i) {
            if (!tracks->pos[i] || !tracks->dir[i]) {
                return fail(DPROP_E_INVALID,
                            "propagate_direct: missing track array");
            }
        }
        if (!tracks->time || !tracks->qop) {
            return fail(DPROP_E_INVALID,
                        "propagate_direct: missing track array");
        }
    }
    if (results->rec_barcode && cfg->max_records == 0u) {
        return fail(DPROP_E_INVALID,
                    "propagate_direct: records need max_records > 0");
    }
    if (n > 0x7fffffffull * k_direct_block) {
        return fail(DPROP_E_INVALID, "propagate_direct: too many tracks");
    }
    const dprop_tracks none{};
    const api::io_ptrs<float> io =
        api::make_io<float>(tracks ? *tracks : none, *results);
    direct_io dio{};
    dio.sequence = seq->barcodes;
    dio.length = seq->length;
    dio.max_length = seq->max_length;
    dio.direction = static_cast<float>(seq->direction);
    dio.start_barcode = seq->start_barcode;
    for (int i = 0; i < 6; ++i) {
        dio.start_bound[i] = seq->start_bound[i];
    }
    const prop_cfg<float> pc = make_prop_cfg<float>(*cfg);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const unsigned int grid =
        static_cast<unsigned int>((n + k_direct_block - 1) / k_direct_block);
    if (det->wires) {
        propagate_direct_kernel<true><<<grid, k_direct_block, 0, st>>>(
            det->view_as<true>(), field->view, pc, io, dio, n);
    } else {
        propagate_direct_kernel<false><<<grid, k_direct_block, 0, st>>>(
            det->view_as<false>(), field->view, pc, io, dio, n);
    }
    DPROP_CUDA(cudaGetLastError());
    return DPROP_OK;
}

}  // extern "C"
