// TEST-ONLY host build of the device propagation core.
//
// The propagation core (detray_b200/csrc/core/*.cuh) is written as
// __host__ __device__ templates.  This file compiles it with the host
// compiler so the tests can compare its navigation and transport logic with
// the reference oracle without a GPU, in double and in float precision.  It
// is not part of the product library and the library never calls it.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "core/config.hpp"
#include "core/convert.hpp"
#include "core/direct.cuh"
#include "core/helix.cuh"
#include "core/phases.cuh"

#include <algorithm>

using namespace dprop;

namespace {
thread_local std::string g_err;

template <typename S>
struct sink_bufs {
    std::vector<S> bound[6];
    std::vector<S> cov[21];
    std::vector<S> path;
};

// Direct-navigation inputs (dprop_sequence with host double arrays)
struct direct_args {
    const uint64_t* barcodes;
    const uint32_t* length;
    uint32_t max_length;
    int32_t direction;
    const uint64_t* start_barcode;
    const double* const* start_bound;
};

template <typename S, bool Grad = false>
int run_g(const dprop_detector_desc* desc, uint32_t field_kind, const double* b,
        const double* lo, const double* hi, const uint32_t* nn,
        const float* values, const dprop_config* c, const double* const* trk,
        uint64_t n, const dprop_results* out, double* tape_rec = nullptr,
        double* tape_init = nullptr, const direct_args* da = nullptr) {
    const std::string problem = validate_desc(desc);
    if (!problem.empty()) {
        g_err = problem;
        return 1;
    }
    const host_tables<S> tables = convert_desc<S>(desc);
    const detector_view<S> det = tables.view();
    field_view<S> f{};
    std::vector<float4> nodes;
    if (field_kind == 0u) {
        f.kind = 0u;
        f.n_r = f.n_phi = f.n_z = 1u;
        for (int i = 0; i < 3; ++i) {
            f.b[i] = static_cast<S>(b[i]);
        }
    } else {
        const uint64_t nn_all = static_cast<uint64_t>(nn[0]) * nn[1] * nn[2];
        nodes.resize(nn_all);
        for (uint64_t i = 0; i < nn_all; ++i) {
            nodes[i] = float4{values[3 * i], values[3 * i + 1],
                              values[3 * i + 2], 0.f};
        }
        f.kind = 1u;
        f.n_r = nn[0];
        f.n_phi = nn[1];
        f.n_z = nn[2];
        f.r_lo = static_cast<S>(lo[0]);
        f.r_step_inv = nn[0] > 1 ? static_cast<S>((nn[0] - 1) / (hi[0] - lo[0])) : S(0);
        f.phi_lo = static_cast<S>(lo[1]);
        f.phi_step_inv = static_cast<S>(nn[1] / (2.0 * constant::pi));
        f.z_lo = static_cast<S>(lo[2]);
        f.z_step_inv = nn[2] > 1 ? static_cast<S>((nn[2] - 1) / (hi[2] - lo[2])) : S(0);
        f.nodes = nodes.data();
    }
    const prop_cfg<S> cfg = make_prop_cfg<S>(*c);
    const uint32_t cap = c->max_records;
    for (uint64_t t = 0; t < n; ++t) {
        nav_cache<S> cache;
        track_state<S, Grad> ts;
        bind_cache(ts.nav, cache);
        bool start_ok = true;
        if (da != nullptr && da->start_barcode != nullptr) {
            S bs[6];
            for (int i = 0; i < 6; ++i) {
                bs[i] = static_cast<S>(da->start_bound[i][t]);
            }
            vec3<S> p{S(0), S(0), S(0)}, d{S(0), S(0), S(1)};
            S tm = S(0), q = bs[4];
            const uint32_t sf = barcode_index(da->start_barcode[t]);
            if (sf < det.n_surfaces) {
                bound_start(det, sf, bs, p, d, tm, q);
            } else {
                start_ok = false;
            }
            init_track_state(ts, p, tm, d, q, cfg);
        } else {
            init_track_state(ts,
                             vec3<S>{static_cast<S>(trk[0][t]), static_cast<S>(trk[1][t]),
                                     static_cast<S>(trk[2][t])},
                             static_cast<S>(trk[3][t]),
                             vec3<S>{static_cast<S>(trk[4][t]), static_cast<S>(trk[5][t]),
                                     static_cast<S>(trk[6][t])},
                             static_cast<S>(trk[7][t]), cfg);
        }
        // records into per-track scratch, then widened into the double outputs
        std::vector<uint64_t> bc(cap);
        std::vector<S> bnd[6], cv[21];
        std::vector<S> pth(cap);
        std::vector<uint8_t> fl(cap);
        record_sink<S> rec{};
        rec.barcode = bc.data();
        S* bptr[6];
        S* cptr[21];
        for (int i = 0; i < 6; ++i) {
            bnd[i].assign(cap, S(0));
            bptr[i] = bnd[i].data();
        }
        for (int i = 0; i < 21; ++i) {
            cv[i].assign(cap, S(0));
            cptr[i] = cv[i].data();
        }
        rec.bound = bptr;
        rec.cov = cptr;
        rec.path = pth.data();
        rec.flags = fl.data();
        rec.n_tracks = 1u;
        rec.track = 0u;
        rec.capacity = cap;
        rec.count = 0u;
        uint8_t status;
        std::vector<S> trec, tinit;
        if (tape_rec != nullptr) {
            // adjoint mode: per-track tape scratch, widened below
            trec.assign(static_cast<size_t>(k_tape_rec) * cap, S(0));
            tinit.assign(k_tape_init, S(0));
            adjoint_tape<S> tape{};
            tape.v.rec = trec.data();
            tape.v.init = tinit.data();
            tape.v.n = 1u;
            tape.v.capacity = cap;
            tape.track = 0u;
            status = propagate_track(ts, det, f, cfg, rec, tape);
            for (int i = 0; i < k_tape_init; ++i) {
                tape_init[static_cast<uint64_t>(i) * n + t] = tinit[i];
            }
            for (int comp = 0; comp < k_tape_rec; ++comp) {
                for (uint32_t k = 0; k < cap; ++k) {
                    tape_rec[(static_cast<uint64_t>(comp) * cap + k) * n + t] =
                        trec[static_cast<size_t>(comp) * cap + k];
                }
            }
        } else if (da != nullptr) {
            ts.nav.direction = static_cast<S>(da->direction);
            direct_navigation<S> navigator;
            navigator.sequence = da->barcodes;
            navigator.n_tracks = n;
            navigator.track = t;
            const uint32_t len = da->length[t];
            navigator.length = static_cast<int32_t>(
                len < da->max_length ? len : da->max_length);
            navigator.next_external = 0;
            navigator.reset(ts.nav, det);
            status = start_ok ? propagate_track_with(navigator, ts, det, f,
                                                     cfg, rec, no_tape{})
                              : uint8_t(DPROP_TRK_NO_SURFACE);
        } else {
            status = propagate_track(ts, det, f, cfg, rec);
        }
        out->status[t] = status;
        if (out->n_records) out->n_records[t] = rec.count;
        if (out->n_steps) out->n_steps[t] = ts.step.n_steps;
        if (out->n_trials) out->n_trials[t] = ts.step.n_trials;
        if (out->n_intersections) out->n_intersections[t] = ts.nav.n_isect;
        if (out->n_transports) out->n_transports[t] = ts.n_transport;
        if (out->n_material) out->n_material[t] = ts.n_material;
        if (out->path_length)
            static_cast<double*>(out->path_length)[t] = ts.step.path_length;
        const double fin[8] = {ts.step.pos.x, ts.step.pos.y, ts.step.pos.z,
                               ts.step.time,  ts.step.dir.x, ts.step.dir.y,
                               ts.step.dir.z, ts.step.qop};
        for (int i = 0; i < 8; ++i) {
            if (out->final_free[i]) static_cast<double*>(out->final_free[i])[t] = fin[i];
        }
        const uint32_t m = rec.count < cap ? rec.count : cap;
        for (uint32_t k = 0; k < m; ++k) {
            const uint64_t o = static_cast<uint64_t>(k) * n + t;
            if (out->rec_barcode) out->rec_barcode[o] = bc[k];
            if (out->rec_flags) out->rec_flags[o] = fl[k];
            if (out->rec_path) static_cast<double*>(out->rec_path)[o] = pth[k];
            for (int i = 0; i < 6; ++i) {
                if (out->rec_bound[i]) static_cast<double*>(out->rec_bound[i])[o] = bnd[i][k];
            }
            for (int i = 0; i < 21; ++i) {
                if (out->rec_cov[i]) static_cast<double*>(out->rec_cov[i])[o] = cv[i][k];
            }
        }
    }
    return 0;
}
template <typename S>
void poison(track_state<S>& ts, loop_state<S>& ls, nav_cache<S>& cache) {
    std::memset(static_cast<void*>(&ts), 0xff, sizeof(ts));
    std::memset(static_cast<void*>(&ls), 0xff, sizeof(ls));
    std::memset(static_cast<void*>(&cache), 0xff, sizeof(cache));
    bind_cache(ts.nav, cache);
}

template <typename S>
field_view<S> host_field(uint32_t field_kind, const double* b,
                         const double* lo, const double* hi,
                         const uint32_t* nn, const float* values,
                         std::vector<float4>& nodes) {
    field_view<S> f{};
    if (field_kind == 0u) {
        f.kind = 0u;
        f.n_r = f.n_phi = f.n_z = 1u;
        for (int i = 0; i < 3; ++i) {
            f.b[i] = static_cast<S>(b[i]);
        }
        return f;
    }
    const uint64_t nn_all = static_cast<uint64_t>(nn[0]) * nn[1] * nn[2];
    nodes.resize(nn_all);
    for (uint64_t i = 0; i < nn_all; ++i) {
        nodes[i] = float4{values[3 * i], values[3 * i + 1], values[3 * i + 2],
                          0.f};
    }
    f.kind = 1u;
    f.n_r = nn[0];
    f.n_phi = nn[1];
    f.n_z = nn[2];
    f.r_lo = static_cast<S>(lo[0]);
    f.r_step_inv =
        nn[0] > 1 ? static_cast<S>((nn[0] - 1) / (hi[0] - lo[0])) : S(0);
    f.phi_lo = static_cast<S>(lo[1]);
    f.phi_step_inv = static_cast<S>(nn[1] / (2.0 * constant::pi));
    f.z_lo = static_cast<S>(lo[2]);
    f.z_step_inv =
        nn[2] > 1 ? static_cast<S>((nn[2] - 1) / (hi[2] - lo[2])) : S(0);
    f.nodes = nodes.data();
    return f;
}

template <typename S, bool W>
int run_rounds_w(const detector_view<S, W>& det, uint32_t field_kind,
                 const double* b, const double* lo, const double* hi,
                 const uint32_t* nn, const float* values,
                 const dprop_config* c, const double* const* trk, uint64_t n,
                 const dprop_results* out, uint32_t rounds,
                 uint32_t step_budget, uint32_t yield_min, uint32_t* stats) {
    std::vector<float4> nodes;
    const field_view<S> f =
        host_field<S>(field_kind, b, lo, hi, nn, values, nodes);
    const prop_cfg<S> cfg = make_prop_cfg<S>(*c);
    const uint32_t cap = c->max_records;
    std::vector<unsigned char> mem(carve_slots<S>(nullptr, n, W, nullptr) + 256);
    slot_soa<S> s{};
    void* base = reinterpret_cast<void*>(
        (reinterpret_cast<uintptr_t>(mem.data()) + 255u) & ~uintptr_t(255u));
    carve_slots<S>(base, n, W, &s);
    // records, slot-major in S; widened at the end
    std::vector<uint64_t> rbc(static_cast<size_t>(cap) * n, 0u);
    std::vector<S> rb[6], rc[21];
    S* bptr[6];
    S* cptr[21];
    for (int i = 0; i < 6; ++i) {
        rb[i].assign(static_cast<size_t>(cap) * n, S(0));
        bptr[i] = rb[i].data();
    }
    for (int i = 0; i < 21; ++i) {
        rc[i].assign(static_cast<size_t>(cap) * n, S(0));
        cptr[i] = rc[i].data();
    }
    std::vector<S> rp(static_cast<size_t>(cap) * n, S(0));
    std::vector<uint8_t> rf(static_cast<size_t>(cap) * n, 0u);
    record_sink<S> rec{};
    rec.barcode = rbc.data();
    rec.bound = bptr;
    rec.cov = cptr;
    rec.path = rp.data();
    rec.flags = rf.data();
    rec.n_tracks = n;
    rec.capacity = cap;
    // records staged per slot as in the kernels, converted at the end; the
    // slots hold the tracks in reverse order so that the conversion's
    // slot -> track mapping is exercised
    std::vector<uint32_t> stage(static_cast<size_t>(cap) * n *
                                    staged_record_words<S>() +
                                4u);
    uint32_t* stage_base = reinterpret_cast<uint32_t*>(
        (reinterpret_cast<uintptr_t>(stage.data()) + 15u) & ~uintptr_t(15u));
    record_sink<S> direct = rec;
    direct.stage = nullptr;
    rec.stage = stage_base;

    auto emit = [&](const track_outputs<S>& o, uint64_t t) {
        out->status[t] = o.status;
        if (out->n_records) out->n_records[t] = o.n_records;
        if (out->n_steps) out->n_steps[t] = o.n_steps;
        if (out->n_trials) out->n_trials[t] = o.n_trials;
        if (out->n_intersections) out->n_intersections[t] = o.n_isect;
        if (out->n_transports) out->n_transports[t] = o.n_transport;
        if (out->n_material) out->n_material[t] = o.n_material;
        if (out->path_length)
            static_cast<double*>(out->path_length)[t] = o.path_length;
        for (int i = 0; i < 8; ++i) {
            if (out->final_free[i])
                static_cast<double*>(out->final_free[i])[t] = o.fin[i];
        }
    };

    for (uint64_t t = 0; t < n; ++t) {
        phase_init<S, W>(s, n - 1u - t, static_cast<uint32_t>(t),
                         vec3<S>{static_cast<S>(trk[0][t]), static_cast<S>(trk[1][t]),
                                 static_cast<S>(trk[2][t])},
                         static_cast<S>(trk[3][t]),
                         vec3<S>{static_cast<S>(trk[4][t]), static_cast<S>(trk[5][t]),
                                 static_cast<S>(trk[6][t])},
                         static_cast<S>(trk[7][t]), det, cfg);
    }
    std::vector<uint64_t> qf, qs, qn;
    for (uint32_t r = 0; r <= rounds; ++r) {
        qf.clear();
        qs.clear();
        qn.clear();
        for (uint64_t slot = 0; slot < n; ++slot) {
            const uint8_t pc = s.pc[slot];
            if (pc == pc_surf) {
                qs.push_back(slot);
            } else if (pc == pc_nav) {
                qn.push_back(slot);
            } else if (pc != pc_done) {
                qf.push_back(slot);
            }
        }
        if (stats != nullptr) {
            stats[3u * r + 0u] = static_cast<uint32_t>(qf.size());
            stats[3u * r + 1u] = static_cast<uint32_t>(qs.size());
            stats[3u * r + 2u] = static_cast<uint32_t>(qn.size());
        }
        if (r == rounds) {
            // tail: everything still alive, every segment inline
            for (uint64_t slot = 0; slot < n; ++slot) {
                if (s.pc[slot] == pc_done) continue;
                const track_outputs<S> o = phase_tail<S, W>(s, slot, det, f, cfg, rec);
                emit(o, s.track[slot]);
            }
            break;
        }
        // fast phase, in groups of 32 queue entries
        for (size_t g0 = 0; g0 < qf.size(); g0 += 32u) {
            const size_t m = (qf.size() - g0) < 32u ? qf.size() - g0 : 32u;
            nav_cache<S> cache[32];
            track_state<S> ts[32];
            loop_state<S> ls[32];
            cand_window c0[32];
            bool active[32];
            for (size_t l = 0; l < m; ++l) {
                poison(ts[l], ls[l], cache[l]);
                fast_load<S, W>(s, qf[g0 + l], ts[l], ls[l], c0[l]);
                active[l] = true;
            }
            for (uint32_t it = 0;; ++it) {
                uint32_t n_active = 0;
                for (size_t l = 0; l < m; ++l) {
                    if (!active[l]) continue;
                    const uint8_t pc = fast_advance<S, W>(
                        ts[l], ls[l], c0[l], s, qf[g0 + l], det, f, cfg, rec);
                    active[l] = machine_is_fast(pc);
                    n_active += active[l] ? 1u : 0u;
                }
                if (n_active == 0u || it + 1u >= step_budget ||
                    n_active < yield_min) {
                    break;
                }
            }
            for (size_t l = 0; l < m; ++l) {
                const uint64_t slot = qf[g0 + l];
                fast_store<S, W>(s, slot, ts[l], ls[l], c0[l]);
                if (ls[l].pc == pc_done) {
                    emit(fast_outputs(s, slot, ts[l], ls[l]), s.track[slot]);
                }
            }
        }
        for (const uint64_t slot : qn) {
            phase_nav<S, W>(s, slot, det, cfg);
        }
    }
    for (uint64_t t = 0; t < n; ++t) {
        const uint64_t slot = n - 1u - t;
        unstage_records<S>(stage_base, slot, s.rec_count[slot], t, direct);
    }
    for (uint64_t t = 0; t < n; ++t) {
        const uint32_t m = out->n_records ? (out->n_records[t] < cap ? out->n_records[t] : cap) : 0u;
        for (uint32_t k = 0; k < m; ++k) {
            const uint64_t o = static_cast<uint64_t>(k) * n + t;
            if (out->rec_barcode) out->rec_barcode[o] = rbc[o];
            if (out->rec_flags) out->rec_flags[o] = rf[o];
            if (out->rec_path) static_cast<double*>(out->rec_path)[o] = rp[o];
            for (int i = 0; i < 6; ++i) {
                if (out->rec_bound[i]) static_cast<double*>(out->rec_bound[i])[o] = rb[i][o];
            }
            for (int i = 0; i < 21; ++i) {
                if (out->rec_cov[i]) static_cast<double*>(out->rec_cov[i])[o] = rc[i][o];
            }
        }
    }
    return 0;
}

// run_g with the transport Jacobian including the field gradient when the
// configuration asks for it (use_field_gradient).
template <typename S>
int run(const dprop_detector_desc* desc, uint32_t field_kind, const double* b,
        const double* lo, const double* hi, const uint32_t* nn,
        const float* values, const dprop_config* c, const double* const* trk,
        uint64_t n, const dprop_results* out, double* tape_rec = nullptr,
        double* tape_init = nullptr, const direct_args* da = nullptr) {
    if (c->use_field_gradient) {
        return run_g<S, true>(desc, field_kind, b, lo, hi, nn, values, c, trk,
                              n, out, tape_rec, tape_init, da);
    }
    return run_g<S, false>(desc, field_kind, b, lo, hi, nn, values, c, trk, n,
                           out, tape_rec, tape_init, da);
}

// The round-based propagation of the phase kernels, simulated on the host
// with the same phase bodies: every round classifies the slots by their next
// segment first (as the queue builder does), then runs the step phase over
// groups of 32 slots with the kernel's yield rule (all lanes of a group stop
// once fewer than yield_min of them are still in the fast phase, or after
// step_budget steps) and the navigation phase.  After
// `rounds` rounds the remaining slots run the tail.  The local state is
// filled with a poison byte before every load, so a segment reading a field
// its phase does not load changes the results.  stats (optional, rounds + 1
// entries per class) receives the queue sizes per round.
template <typename S>
int run_rounds(const dprop_detector_desc* desc, uint32_t field_kind,
               const double* b, const double* lo, const double* hi,
               const uint32_t* nn, const float* values, const dprop_config* c,
               const double* const* trk, uint64_t n, const dprop_results* out,
               uint32_t rounds, uint32_t step_budget, uint32_t yield_min,
               uint32_t* stats) {
    const std::string problem = validate_desc(desc);
    if (!problem.empty()) {
        g_err = problem;
        return 1;
    }
    const host_tables<S> tables = convert_desc<S>(desc);
    bool wires = has_volume_material(desc);
    for (uint32_t i = 0; i < desc->n_surfaces; ++i) {
        wires = wires || desc->surfaces[i].shape == DPROP_SHAPE_LINE ||
                desc->surfaces[i].material_kind != 0u;
    }
    for (uint32_t i = 0; i < desc->n_slabs; ++i) {
        wires = wires || desc->slabs[i].kind == DPROP_MATERIAL_ROD;
    }
    for (uint32_t i = 0; i < desc->n_grids; ++i) {
        wires = wires || desc->grids[i].multi != 0u;
    }
    if (!wires) {
        return run_rounds_w<S, false>(tables.template view_as<false>(),
                                      field_kind, b, lo, hi, nn, values, c,
                                      trk, n, out, rounds, step_budget,
                                      yield_min, stats);
    }
    return run_rounds_w<S, true>(tables.template view_as<true>(), field_kind,
                                 b, lo, hi, nn, values, c, trk, n, out,
                                 rounds, step_budget, yield_min, stats);
}

}  // namespace

extern "C" {
const char* core_host_last_error(void) { return g_err.c_str(); }

int core_host_propagate(int precision_bytes, const dprop_detector_desc* desc,
                        uint32_t field_kind, const double* b, const double* lo,
                        const double* hi, const uint32_t* nn, const float* values,
                        const dprop_config* cfg, const double* const* trk,
                        uint64_t n, const dprop_results* out) {
    if (precision_bytes == 8) {
        return run<double>(desc, field_kind, b, lo, hi, nn, values, cfg, trk, n, out);
    }
    return run<float>(desc, field_kind, b, lo, hi, nn, values, cfg, trk, n, out);
}

// The round-based propagation of the phase kernels (run_rounds above).
int core_host_propagate_rounds(int precision_bytes,
                               const dprop_detector_desc* desc,
                               uint32_t field_kind, const double* b,
                               const double* lo, const double* hi,
                               const uint32_t* nn, const float* values,
                               const dprop_config* cfg,
                               const double* const* trk, uint64_t n,
                               const dprop_results* out, uint32_t rounds,
                               uint32_t step_budget, uint32_t yield_min,
                               uint32_t* stats) {
    if (precision_bytes == 8) {
        return run_rounds<double>(desc, field_kind, b, lo, hi, nn, values, cfg,
                                  trk, n, out, rounds, step_budget, yield_min,
                                  stats);
    }
    return run_rounds<float>(desc, field_kind, b, lo, hi, nn, values, cfg,
                             trk, n, out, rounds, step_budget, yield_min,
                             stats);
}

// Direct-navigation propagation (constant field b): as
// dprop_propagate_direct with host double arrays; trk may be NULL with a
// bound start.
int core_host_propagate_direct(int precision_bytes,
                               const dprop_detector_desc* desc,
                               const double* b, const dprop_config* cfg,
                               const double* const* trk, uint64_t n,
                               const uint64_t* barcodes,
                               const uint32_t* length, uint32_t max_length,
                               int32_t direction,
                               const uint64_t* start_barcode,
                               const double* const* start_bound,
                               const dprop_results* out) {
    const direct_args da{barcodes, length, max_length, direction,
                         start_barcode, start_bound};
    if (precision_bytes == 8) {
        return run<double>(desc, 0u, b, nullptr, nullptr, nullptr, nullptr,
                           cfg, trk, n, out, nullptr, nullptr, &da);
    }
    return run<float>(desc, 0u, b, nullptr, nullptr, nullptr, nullptr, cfg,
                      trk, n, out, nullptr, nullptr, &da);
}

// Helix scan (dprop_helix_scan) with host double arrays, double precision;
// outputs as ref_helix_scan.
int core_host_helix_scan(const dprop_detector_desc* desc, const double* b,
                         const double* const* trk, uint64_t n,
                         double mask_tol, uint32_t cap, uint8_t* status,
                         uint32_t* n_hits, uint64_t* barcode, double* path,
                         double* loc0, double* loc1, uint16_t* vlink) {
    const std::string problem = validate_desc(desc);
    if (!problem.empty()) {
        g_err = problem;
        return 1;
    }
    const host_tables<double> tables = convert_desc<double>(desc);
    const detector_view<double> det = tables.view();
    const root_cfg<double> cfg{unit::um, 1000u, 5000.0 * unit::mm};
    const vec3<double> bf{b[0], b[1], b[2]};
    for (uint64_t t = 0; t < n; ++t) {
        helix<double> h;
        h.init(vec3<double>{trk[0][t], trk[1][t], trk[2][t]},
               vec3<double>{trk[4][t], trk[5][t], trk[6][t]}, trk[7][t], bf);
        std::vector<scan_hit<double>> hits;
        for (uint32_t sf = 0; sf < det.n_surfaces; ++sf) {
            helix_surface_hits(det, sf, h, mask_tol, cfg,
                               [&](const scan_hit<double>& x) {
                                   hits.push_back(x);
                               });
        }
        if (hits.empty()) {
            status[t] = DPROP_SCAN_EMPTY;
            n_hits[t] = 0u;
            continue;
        }
        std::stable_sort(hits.begin(), hits.end(),
                         [](const scan_hit<double>& a,
                            const scan_hit<double>& c) {
                             return std::fabs(a.path) < std::fabs(c.path);
                         });
        size_t kept = hits.size();
        for (size_t k = 0; k < hits.size(); ++k) {
            if (hits[k].volume_link == static_cast<uint16_t>(k_invalid_link)) {
                kept = k + 1u;
                break;
            }
        }
        n_hits[t] = static_cast<uint32_t>(kept);
        if (kept > cap) {
            status[t] = DPROP_SCAN_OVERFLOW;
            continue;
        }
        status[t] = DPROP_SCAN_OK;
        for (size_t k = 0; k < kept; ++k) {
            const uint64_t o = static_cast<uint64_t>(k) * n + t;
            barcode[o] = det.surfaces[hits[k].sf].barcode;
            path[o] = hits[k].path;
            loc0[o] = hits[k].loc0;
            loc1[o] = hits[k].loc1;
            vlink[o] = hits[k].volume_link;
        }
    }
    return 0;
}

// Navigation validation (dprop_validate_navigation) on host arrays: scan
// outputs as core_host_helix_scan, records as core_host_propagate (double).
int core_host_validate(uint64_t n, const uint8_t* scan_status,
                       const uint32_t* n_hits, const uint64_t* truth_bc,
                       const double* truth_path, const uint16_t* truth_vlink,
                       const uint8_t* rec_status, const uint32_t* n_records,
                       const uint64_t* rec_bc, const double* rec_path,
                       uint32_t max_records, double path_tol,
                       uint32_t* n_missed, uint32_t* n_extra) {
    for (uint64_t t = 0; t < n; ++t) {
        const uint32_t nt = scan_status[t] == DPROP_SCAN_OK ? n_hits[t] : 0u;
        const uint32_t nr =
            n_records[t] < max_records ? n_records[t] : max_records;
        compare_trace(truth_bc, truth_path, truth_vlink, nt, rec_bc, rec_path,
                      nr, rec_status[t] == DPROP_TRK_EXITED, n, t, path_tol,
                      n_missed[t], n_extra[t]);
    }
    return 0;
}

// Adjoint-mode propagation: as core_host_propagate, plus the tape
// (tape_rec: [k_tape_rec][max_records][n], tape_init: [k_tape_init][n]).
int core_host_propagate_adjoint(int precision_bytes,
                                const dprop_detector_desc* desc,
                                uint32_t field_kind, const double* b,
                                const double* lo, const double* hi,
                                const uint32_t* nn, const float* values,
                                const dprop_config* cfg,
                                const double* const* trk, uint64_t n,
                                const dprop_results* out, double* tape_rec,
                                double* tape_init) {
    if (tape_rec == nullptr || tape_init == nullptr) {
        g_err = "tape arrays are required";
        return 1;
    }
    if (precision_bytes == 8) {
        return run<double>(desc, field_kind, b, lo, hi, nn, values, cfg, trk,
                           n, out, tape_rec, tape_init);
    }
    return run<float>(desc, field_kind, b, lo, hi, nn, values, cfg, trk, n,
                      out, tape_rec, tape_init);
}

// Reverse sweep over the records of core_host_propagate_adjoint (double
// precision).  grad_bound: 6 slot-major arrays (entries may be NULL);
// grad_free: 8 arrays of n; grad_align: n_surfaces x 6 (accumulated) or NULL.
int core_host_backward(const dprop_detector_desc* desc, uint32_t capacity,
                       const double* const* trk, uint64_t n,
                       const uint32_t* n_records, const uint64_t* rec_barcode,
                       const uint8_t* rec_flags,
                       const double* const* rec_bound, const double* tape_rec,
                       const double* tape_init,
                       const double* const* grad_bound,
                       double* const* grad_free, double* grad_align) {
    const std::string problem = validate_desc(desc);
    if (!problem.empty()) {
        g_err = problem;
        return 1;
    }
    const host_tables<double> tables = convert_desc<double>(desc);
    const detector_view<double> det = tables.view();
    tape_view<double> tp{};
    tp.rec = const_cast<double*>(tape_rec);
    tp.init = const_cast<double*>(tape_init);
    tp.n = n;
    tp.capacity = capacity;
    for (uint64_t t = 0; t < n; ++t) {
        double g[8];
        const vec3<double> dir0{trk[4][t], trk[5][t], trk[6][t]};
        backward_track(det, tp, t, n_records[t], rec_barcode, rec_flags,
                       rec_bound, grad_bound, dir0, g,
                       [&](uint32_t sf, const double* v) {
                           if (grad_align != nullptr) {
                               for (int j = 0; j < 6; ++j) {
                                   grad_align[6u * sf + j] += v[j];
                               }
                           }
                       });
        for (int i = 0; i < 8; ++i) {
            if (grad_free[i] != nullptr) {
                grad_free[i][t] = g[i];
            }
        }
    }
    return 0;
}
}

extern "C" int core_host_field_eval(int precision_bytes, const double* lo,
                                    const double* hi, const uint32_t* nn,
                                    const float* values, const double* xyz,
                                    uint64_t count, double* out) {
    const uint64_t n_all = static_cast<uint64_t>(nn[0]) * nn[1] * nn[2];
    std::vector<float4> nodes(n_all);
    for (uint64_t i = 0; i < n_all; ++i) {
        nodes[i] = float4{values[3 * i], values[3 * i + 1], values[3 * i + 2], 0.f};
    }
    auto run = [&](auto zero) {
        using S = decltype(zero);
        field_view<S> f{};
        f.kind = 1u;
        f.n_r = nn[0];
        f.n_phi = nn[1];
        f.n_z = nn[2];
        f.r_lo = static_cast<S>(lo[0]);
        f.r_step_inv = nn[0] > 1 ? static_cast<S>((nn[0] - 1) / (hi[0] - lo[0])) : S(0);
        f.phi_lo = static_cast<S>(lo[1]);
        f.phi_step_inv = static_cast<S>(nn[1] / (2.0 * constant::pi));
        f.z_lo = static_cast<S>(lo[2]);
        f.z_step_inv = nn[2] > 1 ? static_cast<S>((nn[2] - 1) / (hi[2] - lo[2])) : S(0);
        f.nodes = nodes.data();
        for (uint64_t i = 0; i < count; ++i) {
            const vec3<S> b = field_at(f, vec3<S>{static_cast<S>(xyz[3 * i]),
                                                  static_cast<S>(xyz[3 * i + 1]),
                                                  static_cast<S>(xyz[3 * i + 2])});
            out[3 * i] = b.x;
            out[3 * i + 1] = b.y;
            out[3 * i + 2] = b.z;
        }
    };
    if (precision_bytes == 8) {
        run(0.0);
    } else {
        run(0.0f);
    }
    return 0;
}

// Mean Bethe-Bloch stopping power (energy per length) and its q/p
// derivative of the core's material physics for one slab, in double.
extern "C" int core_host_bethe(const dprop_slab_desc* slab, double mass,
                               double qop, double q, double* dedx,
                               double* ddedx_dqop) {
    const dev_slab<double> s = convert_slab<double>(*slab);
    const rel_quantities<double> rq = make_rq(mass, qop, q);
    const double bb = bethe_bloch(s, rq);
    *dedx = bb;
    *ddedx_dqop = bethe_bloch_dqop(s, rq, bb);
    return 0;
}
