// Magnetic field lookup, field.at(x, y, z).
//
// The stepper queries the field at every RKN stage
// (core/include/detray/propagator/rk_stepper.hpp:338-406).  Two fields are
// supported:
//   * constant (covfie::backend::constant, bfield.hpp:35-40);
//   * a node map on a regular (r, phi, z) grid with linear interpolation in
//     each coordinate and clamping at the edges (the covfie
//     affine<linear<clamp<strided<...>>>> composition of bfield.hpp:43-47,
//     on cylindrical axes; phi periodic, one phi node = axial symmetry).
// Node values are float4 (B_r, B_phi, B_z, 0) so one corner is one 16-byte
// vector load; an axially symmetric lookup touches 4 nodes (2 x 32 bytes
// when the r-neighbours share a sector).
#pragma once

#include "tables.cuh"

namespace dprop {

template <typename S>
DPROP_HD void clamp_locate(S x, S lo, S step_inv, uint32_t n, uint32_t& i0,
                           S& f) {
    if (n < 2u) {
        i0 = 0u;
        f = S(0);
        return;
    }
    S u = (x - lo) * step_inv;
    const S umax = static_cast<S>(n - 1u);
    u = (u >= S(0)) ? u : S(0);  // also maps NaN onto the first node
    u = u > umax ? umax : u;
    S fl = floor(u);
    fl = fl > umax - S(1) ? umax - S(1) : fl;
    i0 = static_cast<uint32_t>(fl);
    f = u - fl;
}

template <typename S>
DPROP_HD float4 load_node(const float4* nodes, uint64_t idx) {
#if defined(__CUDA_ARCH__)
    return __ldg(nodes + idx);
#else
    return nodes[idx];
#endif
}

template <typename S>
DPROP_HD vec3<S> field_at(const field_view<S>& f, vec3<S> p) {
    if (f.kind == 0u) {
        return {f.b[0], f.b[1], f.b[2]};
    }
    const S r = sqrt(p.x * p.x + p.y * p.y);
    uint32_t ir, iz;
    S fr, fz;
    clamp_locate(r, f.r_lo, f.r_step_inv, f.n_r, ir, fr);
    clamp_locate(p.z, f.z_lo, f.z_step_inv, f.n_z, iz, fz);
    const uint32_t ir1 = (f.n_r > 1u) ? ir + 1u : ir;
    const uint32_t iz1 = (f.n_z > 1u) ? iz + 1u : iz;

    uint32_t ip0 = 0u, ip1 = 0u;
    S fp = S(0);
    if (f.n_phi > 1u) {
        const S phi = atan2(p.y, p.x);
        const S nphi = static_cast<S>(f.n_phi);
        S u = (phi - f.phi_lo) * f.phi_step_inv;
        u = u - floor(u / nphi) * nphi;
        const S fl = floor(u);
        ip0 = static_cast<uint32_t>(fl) % f.n_phi;
        ip1 = (ip0 + 1u) % f.n_phi;
        fp = u - fl;
    }
    const uint64_t nr = f.n_r;
    const uint64_t np = f.n_phi;
    auto idx = [&](uint32_t a, uint32_t b, uint32_t c) {
        return (static_cast<uint64_t>(c) * np + b) * nr + a;
    };
    const float4 c000 = load_node<S>(f.nodes, idx(ir, ip0, iz));
    const float4 c100 = load_node<S>(f.nodes, idx(ir1, ip0, iz));
    const float4 c001 = load_node<S>(f.nodes, idx(ir, ip0, iz1));
    const float4 c101 = load_node<S>(f.nodes, idx(ir1, ip0, iz1));
    S b[3];
    const float* a000 = &c000.x;
    const float* a100 = &c100.x;
    const float* a001 = &c001.x;
    const float* a101 = &c101.x;
    if (f.n_phi > 1u) {
        const float4 c010 = load_node<S>(f.nodes, idx(ir, ip1, iz));
        const float4 c110 = load_node<S>(f.nodes, idx(ir1, ip1, iz));
        const float4 c011 = load_node<S>(f.nodes, idx(ir, ip1, iz1));
        const float4 c111 = load_node<S>(f.nodes, idx(ir1, ip1, iz1));
        const float* a010 = &c010.x;
        const float* a110 = &c110.x;
        const float* a011 = &c011.x;
        const float* a111 = &c111.x;
        for (int c = 0; c < 3; ++c) {
            const S c00 = S(a000[c]) + fr * (S(a100[c]) - S(a000[c]));
            const S c10 = S(a010[c]) + fr * (S(a110[c]) - S(a010[c]));
            const S c01 = S(a001[c]) + fr * (S(a101[c]) - S(a001[c]));
            const S c11 = S(a011[c]) + fr * (S(a111[c]) - S(a011[c]));
            const S c0 = c00 + fp * (c10 - c00);
            const S c1 = c01 + fp * (c11 - c01);
            b[c] = c0 + fz * (c1 - c0);
        }
    } else {
        for (int c = 0; c < 3; ++c) {
            const S c0 = S(a000[c]) + fr * (S(a100[c]) - S(a000[c]));
            const S c1 = S(a001[c]) + fr * (S(a101[c]) - S(a001[c]));
            b[c] = c0 + fz * (c1 - c0);
        }
    }
    const S cp = (r > S(0)) ? p.x / r : S(1);
    const S sp = (r > S(0)) ? p.y / r : S(0);
    return {b[0] * cp - b[1] * sp, b[0] * sp + b[1] * cp, b[2]};
}

}  // namespace dprop
