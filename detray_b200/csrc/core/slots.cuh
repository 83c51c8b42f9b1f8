// Per-track state of the round-based propagation, kept in device memory
// between the phase kernels: one array per scalar field, indexed by the
// track's slot (its position in the direction-sorted batch), so that the
// lanes of a warp working on neighbouring slots read and write neighbouring
// words.
//
// Each kernel loads and stores only the field groups its segments touch:
//   step   the stepper state (rk_stepper::state): position, direction, q/p,
//          time, path lengths, step sizes, dt/ds, constraint, the 25 free
//          transport-Jacobian entries, trial and step counters
//   meta   navigation state without the candidates: cache indices, status,
//          trust, volume, external mask tolerance, direction, abort reason,
//          intersection counter
//   cand   the candidate cache, the k_cache + 1 entries of a slot stored
//          together (one 16-byte record each), so that the few entries a
//          lane reads at its own run-time cache index share a cache line: a
//          phase loads only the entries it reads (the step phase the current
//          surface, the target and the one after it, the navigation phase
//          all of them)
//   bound  bound parameters, covariance and surface of the transporter
//   loop   loop variables (iteration, stall counter, path before the step,
//          flags, charge)
//   count  transport/material counters, record count, input index
//   cyc    the exact-cycle search (detectors with wire surfaces)
//   pc     the next segment of each slot, one byte per slot in its own dense
//          array (the queue builder reads only this)
#pragma once

#include <cstring>

#include "machine.cuh"

namespace dprop {

// Slots per tile of the queue builder; the next-segment array is padded to a
// whole number of tiles.
constexpr uint64_t k_queue_tile = 4096u;

DPROP_HD uint64_t queue_tiles(uint64_t n) {
    return (n + k_queue_tile - 1u) / k_queue_tile;
}

enum slot_group : uint32_t {
    g_free = 1u,      // position, direction, q/p, time
    g_jac = 2u,       // the free transport Jacobian
    g_pathdtds = 4u,  // signed path length, dt/ds
    g_stepctl = 8u,   // absolute path, step sizes, constraint, counters
    g_meta = 16u,
    g_bound = 32u,
    g_loop = 64u,
    g_count = 128u,   // transport and material counters
    g_cyc = 256u,
    g_step = g_free | g_jac | g_pathdtds | g_stepctl,
};

template <typename S>
struct slot_soa {
    uint64_t n;  // slots (row stride of the per-candidate arrays)
    // step
    S* pos[3];
    S* dir[3];
    S* qop;
    S* time;
    double* path_length;
    double* abs_path_length;
    S* step_size;
    S* next_step_size;
    S* constraint;
    S* dtds[3];
    S* jac[25];  // A (9, row-major), B (9), c (3), d (3), e
    uint32_t* n_trials;
    uint32_t* n_steps;
    // meta
    uint32_t* nav_bytes;  // next | last << 8 | status << 16 | trust << 24
    uint32_t* volume;
    S* external_tol;
    S* direction;
    uint32_t* nav_misc;   // abort reason
    uint32_t* n_isect;
    // cand: record k of slot s at [s * (k_cache + 1) + k]; float: path bits,
    // surface, info, 0; double: path bits (low, high), surface, info; info
    // = volume_link | status << 16 | flags << 24
    uint4* cand;
    // bound
    S* bv[6];
    S* bcov[21];
    uint32_t* bsf;
    // loop
    double* path_prev;
    uint32_t* iter;
    uint32_t* stall;
    uint32_t* flags;  // heartbeat | is_init << 1 | out_of_budget << 2 |
                      // nav_mode << 3 | (q < 0) << 4
    // count
    uint32_t* n_transport;
    uint32_t* n_material;
    uint32_t* rec_count;
    uint32_t* track;
    // cyc
    uint32_t* cyc_u[5];  // key, lam, power, period, hits
    double* cyc_abs0;
    double* cyc_path0;
    S* cyc_time0;
    // dense next-segment array
    uint8_t* pc;
};

// The arrays of n slots carved out of one block of device memory, each
// rounded up to 256 bytes.  With base == 0 nothing is written and the
// return value is the size the block needs.
template <typename S>
size_t carve_slots(void* base, uint64_t n, bool with_cyc, slot_soa<S>* out) {
    uintptr_t p = reinterpret_cast<uintptr_t>(base);
    const uintptr_t p0 = p;
    auto take = [&p](size_t b) {
        const uintptr_t r = p;
        p += (b + 255u) & ~size_t(255u);
        return r;
    };
    auto fs = [&]() { return reinterpret_cast<S*>(take(n * sizeof(S))); };
    auto f4 = [&]() { return reinterpret_cast<uint32_t*>(take(n * 4u)); };
    auto f8 = [&]() { return reinterpret_cast<double*>(take(n * 8u)); };
    slot_soa<S> s{};
    s.n = n;
    for (int i = 0; i < 3; ++i) s.pos[i] = fs();
    for (int i = 0; i < 3; ++i) s.dir[i] = fs();
    s.qop = fs();
    s.time = fs();
    s.path_length = f8();
    s.abs_path_length = f8();
    s.step_size = fs();
    s.next_step_size = fs();
    s.constraint = fs();
    for (int i = 0; i < 3; ++i) s.dtds[i] = fs();
    for (int i = 0; i < 25; ++i) s.jac[i] = fs();
    s.n_trials = f4();
    s.n_steps = f4();
    s.nav_bytes = f4();
    s.volume = f4();
    s.external_tol = fs();
    s.direction = fs();
    s.nav_misc = f4();
    s.n_isect = f4();
    s.cand = reinterpret_cast<uint4*>(
        take(static_cast<size_t>(k_cache + 1) * n * sizeof(uint4)));
    for (int i = 0; i < 6; ++i) s.bv[i] = fs();
    for (int i = 0; i < 21; ++i) s.bcov[i] = fs();
    s.bsf = f4();
    s.path_prev = f8();
    s.iter = f4();
    s.stall = f4();
    s.flags = f4();
    s.n_transport = f4();
    s.n_material = f4();
    s.rec_count = f4();
    s.track = f4();
    if (with_cyc) {
        for (int i = 0; i < 5; ++i) s.cyc_u[i] = f4();
        s.cyc_abs0 = f8();
        s.cyc_path0 = f8();
        s.cyc_time0 = fs();
    }
    s.pc = reinterpret_cast<uint8_t*>(take(queue_tiles(n) * k_queue_tile));
    if (out != nullptr) {
        *out = s;
    }
    return static_cast<size_t>(p - p0);
}

// ----------------------------------------------------------- candidates
DPROP_HD uint32_t f32_bits(float v) {
    uint32_t u;
    memcpy(&u, &v, sizeof(u));
    return u;
}
DPROP_HD float bits_f32(uint32_t u) {
    float v;
    memcpy(&v, &u, sizeof(v));
    return v;
}

DPROP_HD void pack_path(float p, uint4& r) {
    r.x = f32_bits(p);
    r.w = 0u;
}
DPROP_HD void pack_path(double p, uint4& r) {
    uint64_t u;
    memcpy(&u, &p, sizeof(u));
    r.x = static_cast<uint32_t>(u);
    r.w = static_cast<uint32_t>(u >> 32);
}
DPROP_HD void unpack_path(const uint4& r, float& p) { p = bits_f32(r.x); }
DPROP_HD void unpack_path(const uint4& r, double& p) {
    const uint64_t u = static_cast<uint64_t>(r.x) |
                       (static_cast<uint64_t>(r.w) << 32);
    memcpy(&p, &u, sizeof(p));
}

template <typename S>
DPROP_HD void load_cand(const slot_soa<S>& s, uint64_t slot, int k,
                        candidate<S>& c) {
    const uint4 r = s.cand[slot * static_cast<uint64_t>(k_cache + 1) +
                           static_cast<uint64_t>(k)];
    unpack_path(r, c.path);
    c.sf = r.y;
    c.volume_link = static_cast<uint16_t>(r.z & 0xffffu);
    c.status = static_cast<uint8_t>((r.z >> 16) & 0xffu);
    c.flags = static_cast<uint8_t>(r.z >> 24);
}

template <typename S>
DPROP_HD void store_cand(const slot_soa<S>& s, uint64_t slot, int k,
                         const candidate<S>& c) {
    uint4 r;
    pack_path(c.path, r);
    r.y = c.sf;
    r.z = static_cast<uint32_t>(c.volume_link) |
          (static_cast<uint32_t>(c.status) << 16) |
          (static_cast<uint32_t>(c.flags) << 24);
    s.cand[slot * static_cast<uint64_t>(k_cache + 1) +
           static_cast<uint64_t>(k)] = r;
}

// Candidate indices [lo, hi] clamped to the cache (including its sentinel).
DPROP_HD void cand_range(int a, int b, int& lo, int& hi) {
    lo = a < 0 ? 0 : a;
    hi = b > k_cache ? k_cache : b;
}

// ------------------------------------------------------------- groups
template <typename S, typename LS>
DPROP_HD void load_slot(const slot_soa<S>& s, uint64_t slot, uint32_t groups,
                        track_state<S>& ts, LS& ls) {
    step_state<S>& st = ts.step;
    if (groups & g_free) {
        st.pos = {s.pos[0][slot], s.pos[1][slot], s.pos[2][slot]};
        st.dir = {s.dir[0][slot], s.dir[1][slot], s.dir[2][slot]};
        st.qop = s.qop[slot];
        st.time = s.time[slot];
    }
    if (groups & g_jac) {
        for (int i = 0; i < 9; ++i) st.jac.A.m[i] = s.jac[i][slot];
        for (int i = 0; i < 9; ++i) st.jac.B.m[i] = s.jac[9 + i][slot];
        st.jac.c = {s.jac[18][slot], s.jac[19][slot], s.jac[20][slot]};
        st.jac.d = {s.jac[21][slot], s.jac[22][slot], s.jac[23][slot]};
        st.jac.e = s.jac[24][slot];
    }
    if (groups & g_pathdtds) {
        st.path_length = s.path_length[slot];
        st.dtds = {s.dtds[0][slot], s.dtds[1][slot], s.dtds[2][slot]};
        st.dqopds = S(0);
    }
    if (groups & g_stepctl) {
        st.abs_path_length = s.abs_path_length[slot];
        st.step_size = s.step_size[slot];
        st.next_step_size = s.next_step_size[slot];
        st.constraint = s.constraint[slot];
        st.n_trials = s.n_trials[slot];
        st.n_steps = s.n_steps[slot];
    }
    if (groups & g_meta) {
        nav_state<S>& nav = ts.nav;
        const uint32_t b = s.nav_bytes[slot];
        nav.next = static_cast<int8_t>(b & 0xffu);
        nav.last = static_cast<int8_t>((b >> 8) & 0xffu);
        nav.status = static_cast<int8_t>((b >> 16) & 0xffu);
        nav.trust = static_cast<uint8_t>(b >> 24);
        nav.volume = s.volume[slot];
        nav.external_tol = s.external_tol[slot];
        nav.direction = s.direction[slot];
        nav.reason = static_cast<uint8_t>(s.nav_misc[slot]);
        nav.n_isect = s.n_isect[slot];
    }
    if (groups & g_bound) {
        for (int i = 0; i < 6; ++i) ts.bound.v[i] = s.bv[i][slot];
        for (int i = 0; i < 21; ++i) ts.bound.cov[i] = s.bcov[i][slot];
        ts.bound.sf = s.bsf[slot];
    }
    if (groups & g_loop) {
        ls.path_prev = s.path_prev[slot];
        ls.i = s.iter[slot];
        ls.stall = s.stall[slot];
        const uint32_t f = s.flags[slot];
        ts.heartbeat = (f & 1u) != 0u;
        ls.is_init = (f & 2u) != 0u;
        ls.out_of_budget = (f & 4u) != 0u;
        ls.nav_mode = static_cast<uint8_t>((f >> 3) & 1u);
        ts.q = (f & 16u) ? S(-1) : S(1);
    }
    if (groups & g_count) {
        ts.n_transport = s.n_transport[slot];
        ts.n_material = s.n_material[slot];
    }
    if (groups & g_cyc) {
        ls.cyc.key = s.cyc_u[0][slot];
        ls.cyc.lam = s.cyc_u[1][slot];
        ls.cyc.power = s.cyc_u[2][slot];
        ls.cyc.period = s.cyc_u[3][slot];
        ls.cyc.hits = s.cyc_u[4][slot];
        ls.cyc.abs0 = s.cyc_abs0[slot];
        ls.cyc.path0 = s.cyc_path0[slot];
        ls.cyc.time0 = s.cyc_time0[slot];
    }
}

template <typename S, typename LS>
DPROP_HD void store_slot(const slot_soa<S>& s, uint64_t slot, uint32_t groups,
                         const track_state<S>& ts, const LS& ls) {
    const step_state<S>& st = ts.step;
    if (groups & g_free) {
        s.pos[0][slot] = st.pos.x;
        s.pos[1][slot] = st.pos.y;
        s.pos[2][slot] = st.pos.z;
        s.dir[0][slot] = st.dir.x;
        s.dir[1][slot] = st.dir.y;
        s.dir[2][slot] = st.dir.z;
        s.qop[slot] = st.qop;
        s.time[slot] = st.time;
    }
    if (groups & g_pathdtds) {
        s.path_length[slot] = st.path_length;
        s.dtds[0][slot] = st.dtds.x;
        s.dtds[1][slot] = st.dtds.y;
        s.dtds[2][slot] = st.dtds.z;
    }
    if (groups & g_stepctl) {
        s.abs_path_length[slot] = st.abs_path_length;
        s.step_size[slot] = st.step_size;
        s.next_step_size[slot] = st.next_step_size;
        s.constraint[slot] = st.constraint;
        s.n_trials[slot] = st.n_trials;
        s.n_steps[slot] = st.n_steps;
    }
    if (groups & g_jac) {
        for (int i = 0; i < 9; ++i) s.jac[i][slot] = st.jac.A.m[i];
        for (int i = 0; i < 9; ++i) s.jac[9 + i][slot] = st.jac.B.m[i];
        s.jac[18][slot] = st.jac.c.x;
        s.jac[19][slot] = st.jac.c.y;
        s.jac[20][slot] = st.jac.c.z;
        s.jac[21][slot] = st.jac.d.x;
        s.jac[22][slot] = st.jac.d.y;
        s.jac[23][slot] = st.jac.d.z;
        s.jac[24][slot] = st.jac.e;
    }
    if (groups & g_meta) {
        const nav_state<S>& nav = ts.nav;
        s.nav_bytes[slot] = static_cast<uint32_t>(static_cast<uint8_t>(nav.next)) |
                            (static_cast<uint32_t>(static_cast<uint8_t>(nav.last)) << 8) |
                            (static_cast<uint32_t>(static_cast<uint8_t>(nav.status)) << 16) |
                            (static_cast<uint32_t>(nav.trust) << 24);
        s.volume[slot] = nav.volume;
        s.external_tol[slot] = nav.external_tol;
        s.direction[slot] = nav.direction;
        s.nav_misc[slot] = nav.reason;
        s.n_isect[slot] = nav.n_isect;
    }
    if (groups & g_bound) {
        for (int i = 0; i < 6; ++i) s.bv[i][slot] = ts.bound.v[i];
        for (int i = 0; i < 21; ++i) s.bcov[i][slot] = ts.bound.cov[i];
        s.bsf[slot] = ts.bound.sf;
    }
    if (groups & g_loop) {
        s.path_prev[slot] = ls.path_prev;
        s.iter[slot] = ls.i;
        s.stall[slot] = ls.stall;
        s.flags[slot] = (ts.heartbeat ? 1u : 0u) | (ls.is_init ? 2u : 0u) |
                        (ls.out_of_budget ? 4u : 0u) |
                        (static_cast<uint32_t>(ls.nav_mode & 1u) << 3) |
                        (ts.q < S(0) ? 16u : 0u);
    }
    if (groups & g_count) {
        s.n_transport[slot] = ts.n_transport;
        s.n_material[slot] = ts.n_material;
    }
    if (groups & g_cyc) {
        s.cyc_u[0][slot] = ls.cyc.key;
        s.cyc_u[1][slot] = ls.cyc.lam;
        s.cyc_u[2][slot] = ls.cyc.power;
        s.cyc_u[3][slot] = ls.cyc.period;
        s.cyc_u[4][slot] = ls.cyc.hits;
        s.cyc_abs0[slot] = ls.cyc.abs0;
        s.cyc_path0[slot] = ls.cyc.path0;
        s.cyc_time0[slot] = ls.cyc.time0;
    }
}

}  // namespace dprop
