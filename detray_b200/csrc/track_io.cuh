// Inputs and outputs of the propagation kernels and the per-track driver
// shared by the kernels of dprop_api.cu and adjoint_api.cu.
#pragma once

#include "api_common.cuh"

namespace dprop::api {

// Device pointers of the inputs/outputs, by value into the kernels: In is
// the element type of the track inputs, S the arithmetic and result type.
template <typename In, typename S = float>
struct io_ptrs {
    const In* trk[8];
    uint8_t* status;
    uint32_t* n_records;
    uint32_t* n_steps;
    uint32_t* n_trials;
    S* path_length;
    S* final_free[8];
    uint64_t* rec_barcode;
    S* rec_bound[6];
    S* rec_cov[21];
    S* rec_path;
    uint8_t* rec_flags;
    uint32_t* n_isect;
    uint32_t* n_transport;
    uint32_t* n_material;
};

template <typename In, typename S = float>
io_ptrs<In, S> make_io(const dprop_tracks& t, const dprop_results& r) {
    io_ptrs<In, S> io{};
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
    io.path_length = static_cast<S*>(r.path_length);
    for (int i = 0; i < 8; ++i) {
        io.final_free[i] = static_cast<S*>(r.final_free[i]);
    }
    io.rec_barcode = r.rec_barcode;
    for (int i = 0; i < 6; ++i) {
        io.rec_bound[i] = static_cast<S*>(r.rec_bound[i]);
    }
    for (int i = 0; i < 21; ++i) {
        io.rec_cov[i] = static_cast<S*>(r.rec_cov[i]);
    }
    io.rec_path = static_cast<S*>(r.rec_path);
    io.rec_flags = r.rec_flags;
    io.n_isect = r.n_intersections;
    io.n_transport = r.n_transports;
    io.n_material = r.n_material;
    return io;
}

// One track from its inputs to its results, in arithmetic type S.  With
// Adjoint the propagation also writes the derivative tape of track t
// (adjoint.cuh); with Grad the transport Jacobian includes the field
// gradient.
template <typename In, bool Adjoint = false, typename S = float, bool W,
          bool Grad = false>
__device__ __forceinline__ void run_one(uint64_t t, uint64_t n,
                                        const detector_view<S, W>& det,
                                        const field_view<S>& field,
                                        const prop_cfg<S>& cfg,
                                        const io_ptrs<In, S>& io,
                                        const tape_view<S>& tv = {}) {
    const vec3<S> pos{static_cast<S>(io.trk[0][t]),
                      static_cast<S>(io.trk[1][t]),
                      static_cast<S>(io.trk[2][t])};
    const vec3<S> dir{static_cast<S>(io.trk[4][t]),
                      static_cast<S>(io.trk[5][t]),
                      static_cast<S>(io.trk[6][t])};
    const S time = static_cast<S>(io.trk[3][t]);
    const S qop = static_cast<S>(io.trk[7][t]);

    nav_cache<S> cache;
    track_state<S, Grad> ts;
    bind_cache(ts.nav, cache);
    init_track_state(ts, pos, time, dir, qop, cfg);

    record_sink<S> rec;
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

    uint8_t status;
    if constexpr (Adjoint) {
        adjoint_tape<S> tape;
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
    if (io.path_length) io.path_length[t] = static_cast<S>(ts.step.path_length);
    const S fin[8] = {ts.step.pos.x, ts.step.pos.y, ts.step.pos.z,
                      ts.step.time,  ts.step.dir.x, ts.step.dir.y,
                      ts.step.dir.z, ts.step.qop};
    for (int i = 0; i < 8; ++i) {
        if (io.final_free[i]) io.final_free[i][t] = fin[i];
    }
}

// Round-based propagation (rounds_api.cu): device scratch bytes for n
// tracks, and the enqueue of the whole propagation on a stream (no
// allocation, no synchronisation; order is the direction-sorted track order
// or NULL).  rec_cap: records per track staged in the scratch (0 when no
// records are requested, see staged_capacity).
size_t rounds_scratch_bytes(uint64_t n, bool wires, uint32_t rec_cap);
size_t rounds_scratch_bytes_fp64(uint64_t n, bool wires, uint32_t rec_cap);

// Records per track the round-based propagation stages in its scratch: the
// configuration's capacity when the caller asks for records.
template <typename S, typename In, typename O>
uint32_t staged_capacity(const prop_cfg<S>& cfg, const io_ptrs<In, O>& io) {
    return io.rec_barcode != nullptr ? cfg.max_records : 0u;
}

// mark: optional event recorded on the stream after round mark_round's
// phase kernels (a later propagation can start then, in the tail of this
// one); NULL: none.
template <typename In>
dprop_status enqueue_rounds(const dprop_launch* lc, const dprop_detector* det,
                            const dprop_field* field,
                            const prop_cfg<float>& cfg, const io_ptrs<In>& io,
                            uint64_t n, const uint32_t* order, void* scratch,
                            size_t scratch_bytes, cudaStream_t stream,
                            cudaEvent_t mark = nullptr,
                            uint32_t mark_round = 0u);

// The same in double precision end to end (dprop_launch.precision = 8).
dprop_status enqueue_rounds_fp64(const dprop_launch* lc,
                                 const dprop_detector* det,
                                 const dprop_field* field,
                                 const prop_cfg<double>& cfg,
                                 const io_ptrs<double, double>& io,
                                 uint64_t n, const uint32_t* order,
                                 void* scratch, size_t scratch_bytes,
                                 cudaStream_t stream);

}  // namespace dprop::api
