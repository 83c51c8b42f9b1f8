// Inputs and outputs of the propagation kernels and the per-track driver
// shared by the kernels of dprop_api.cu and adjoint_api.cu.
#pragma once

#include "api_common.cuh"

namespace dprop::api {

// Device pointers of the inputs/outputs, by value into the kernels
template <typename In>
struct io_ptrs {
    const In* trk[8];
    uint8_t* status;
    uint32_t* n_records;
    uint32_t* n_steps;
    uint32_t* n_trials;
    float* path_length;
    float* final_free[8];
    uint64_t* rec_barcode;
    float* rec_bound[6];
    float* rec_cov[21];
    float* rec_path;
    uint8_t* rec_flags;
    uint32_t* n_isect;
    uint32_t* n_transport;
    uint32_t* n_material;
};

template <typename In>
io_ptrs<In> make_io(const dprop_tracks& t, const dprop_results& r) {
    io_ptrs<In> io{};
    for (int i = 0; i < 3; ++i) {
        io.trk[i] = static_cast<const In*>(t.pos[i]);
        io.trk[4 + i] = static_cast<const In*>(t.dir[i]);
    }
    io.trk[3] = static_cast<const In*>(t.time);
    io.trk[7] = static_cast<const In*>(t.qop);
    io.status = r.status;
    io.n_records = r.n_records;
    io.n_steps = r.n_steps;
    io.n_trials = r.n_trials;
    io.path_length = static_cast<float*>(r.path_length);
    for (int i = 0; i < 8; ++i) {
        io.final_free[i] = static_cast<float*>(r.final_free[i]);
    }
    io.rec_barcode = r.rec_barcode;
    for (int i = 0; i < 6; ++i) {
        io.rec_bound[i] = static_cast<float*>(r.rec_bound[i]);
    }
    for (int i = 0; i < 21; ++i) {
        io.rec_cov[i] = static_cast<float*>(r.rec_cov[i]);
    }
    io.rec_path = static_cast<float*>(r.rec_path);
    io.rec_flags = r.rec_flags;
    io.n_isect = r.n_intersections;
    io.n_transport = r.n_transports;
    io.n_material = r.n_material;
    return io;
}

// One track from its inputs to its results.  With Adjoint the propagation
// also writes the derivative tape of track t (adjoint.cuh).
template <typename In, bool Adjoint = false>
__device__ __forceinline__ void run_one(uint64_t t, uint64_t n,
                                        const detector_view<float>& det,
                                        const field_view<float>& field,
                                        const prop_cfg<float>& cfg,
                                        const io_ptrs<In>& io,
                                        const tape_view<float>& tv = {}) {
    const vec3<float> pos{static_cast<float>(io.trk[0][t]),
                          static_cast<float>(io.trk[1][t]),
                          static_cast<float>(io.trk[2][t])};
    const vec3<float> dir{static_cast<float>(io.trk[4][t]),
                          static_cast<float>(io.trk[5][t]),
                          static_cast<float>(io.trk[6][t])};
    const float time = static_cast<float>(io.trk[3][t]);
    const float qop = static_cast<float>(io.trk[7][t]);

    track_state<float> ts;
    init_track_state(ts, pos, time, dir, qop, cfg);

    record_sink<float> rec;
    rec.barcode = io.rec_barcode;
    for (int i = 0; i < 6; ++i) {
        rec.bound[i] = io.rec_bound[i];
    }
    for (int i = 0; i < 21; ++i) {
        rec.cov[i] = io.rec_cov[i];
    }
    rec.path = io.rec_path;
    rec.flags = io.rec_flags;
    rec.n_tracks = n;
    rec.track = t;
    rec.capacity = (io.rec_barcode != nullptr) ? cfg.max_records : 0u;
    rec.count = 0u;

    uint8_t status;
    if constexpr (Adjoint) {
        adjoint_tape<float> tape;
        tape.v = tv;
        tape.track = t;
        status = propagate_track(ts, det, field, cfg, rec, tape);
    } else {
        status = propagate_track(ts, det, field, cfg, rec);
    }

    if (io.status) io.status[t] = status;
    if (io.n_records) io.n_records[t] = rec.count;
    if (io.n_steps) io.n_steps[t] = ts.step.n_steps;
    if (io.n_trials) io.n_trials[t] = ts.step.n_trials;
    if (io.n_isect) io.n_isect[t] = ts.nav.n_isect;
    if (io.n_transport) io.n_transport[t] = ts.n_transport;
    if (io.n_material) io.n_material[t] = ts.n_material;
    if (io.path_length) io.path_length[t] = static_cast<float>(ts.step.path_length);
    const float fin[8] = {ts.step.pos.x, ts.step.pos.y, ts.step.pos.z,
                          ts.step.time,  ts.step.dir.x, ts.step.dir.y,
                          ts.step.dir.z, ts.step.qop};
    for (int i = 0; i < 8; ++i) {
        if (io.final_free[i]) io.final_free[i][t] = fin[i];
    }
}

}  // namespace dprop::api
