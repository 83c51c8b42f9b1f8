/*
 * ORACLE — test infrastructure only (see ref_harness.cpp).
 *
 * Magnetic field seen by the reference propagator in the oracle build.  The
 * reference plugs a covfie field view into rk_stepper (field.at(x, y, z),
 * core/include/detray/propagator/rk_stepper.hpp:338-344); covfie is not
 * available here, so this class provides the two fields of the benchmark
 * configurations:
 *   - constant: covfie::backend::constant semantics
 *     (tests/include/detray/test/common/bfield.hpp:35-40);
 *   - a map on a regular (r, phi, z) node grid holding (B_r, B_phi, B_z),
 *     interpolated linearly in each coordinate with clamping at the edges
 *     (the covfie linear<clamp<...>> composition of bfield.hpp:43-47, applied
 *     on cylindrical axes).  phi is periodic; with one phi node the map is
 *     axially symmetric.  Evaluated in double from the float node values.
 * The device field of the product implements the same definition.
 */
#pragma once

#include <cmath>
#include <cstdint>

namespace oracle_field {

struct field {
    int kind{0};
    double b[3]{0., 0., 0.};
    double lo[3]{0., 0., 0.};
    double hi[3]{0., 0., 0.};
    uint32_t n[3]{1u, 1u, 1u};
    const float* values{nullptr};

    void set_constant(double bx, double by, double bz) {
        kind = 0;
        b[0] = bx;
        b[1] = by;
        b[2] = bz;
    }
    void set_grid(const double* l, const double* h, const uint32_t* nn,
                  const float* v) {
        kind = 1;
        for (int i = 0; i < 3; ++i) {
            lo[i] = l[i];
            hi[i] = h[i];
            n[i] = nn[i];
        }
        values = v;
    }

    // node value, component c
    double node(uint32_t ir, uint32_t iphi, uint32_t iz, int c) const {
        const uint64_t idx =
            (static_cast<uint64_t>(iz) * n[1] + iphi) * n[0] + ir;
        return static_cast<double>(values[idx * 3u + static_cast<uint64_t>(c)]);
    }

    // clamp a coordinate onto the node axis: lower node and fraction
    static void locate(double x, double l, double h, uint32_t nn,
                       uint32_t& i0, double& f) {
        if (nn < 2u) {
            i0 = 0u;
            f = 0.;
            return;
        }
        const double step = (h - l) / static_cast<double>(nn - 1u);
        double u = (x - l) / step;
        if (u < 0.) {
            u = 0.;
        }
        const double umax = static_cast<double>(nn - 1u);
        if (u > umax) {
            u = umax;
        }
        double fl = std::floor(u);
        if (fl > umax - 1.) {
            fl = umax - 1.;
        }
        i0 = static_cast<uint32_t>(fl);
        f = u - fl;
    }

    void at(double x, double y, double z, double* out) const {
        if (kind == 0) {
            out[0] = b[0];
            out[1] = b[1];
            out[2] = b[2];
            return;
        }
        if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z)) {
            // a non-finite position (the reference continues after a
            // particle stopped in material): no node lookup
            out[0] = out[1] = out[2] = std::nan("");
            return;
        }
        const double r = std::sqrt(x * x + y * y);
        const double phi = std::atan2(y, x);
        uint32_t ir, iz;
        double fr, fz;
        locate(r, lo[0], hi[0], n[0], ir, fr);
        locate(z, lo[2], hi[2], n[2], iz, fz);
        // periodic phi axis: n[1] nodes over [lo, lo + 2 pi)
        uint32_t ip0 = 0u, ip1 = 0u;
        double fp = 0.;
        if (n[1] > 1u) {
            const double two_pi = 6.283185307179586476925286766559;
            const double step = two_pi / static_cast<double>(n[1]);
            double u = (phi - lo[1]) / step;
            u = u - std::floor(u / static_cast<double>(n[1])) *
                        static_cast<double>(n[1]);
            const double fl = std::floor(u);
            ip0 = static_cast<uint32_t>(fl) % n[1];
            ip1 = (ip0 + 1u) % n[1];
            fp = u - fl;
        }
        const uint32_t ir1 = (n[0] > 1u) ? ir + 1u : ir;
        const uint32_t iz1 = (n[2] > 1u) ? iz + 1u : iz;
        double bc[3];
        for (int c = 0; c < 3; ++c) {
            const double c000 = node(ir, ip0, iz, c);
            const double c100 = node(ir1, ip0, iz, c);
            const double c010 = node(ir, ip1, iz, c);
            const double c110 = node(ir1, ip1, iz, c);
            const double c001 = node(ir, ip0, iz1, c);
            const double c101 = node(ir1, ip0, iz1, c);
            const double c011 = node(ir, ip1, iz1, c);
            const double c111 = node(ir1, ip1, iz1, c);
            const double c00 = c000 + fr * (c100 - c000);
            const double c10 = c010 + fr * (c110 - c010);
            const double c01 = c001 + fr * (c101 - c001);
            const double c11 = c011 + fr * (c111 - c011);
            const double c0 = c00 + fp * (c10 - c00);
            const double c1 = c01 + fp * (c11 - c01);
            bc[c] = c0 + fz * (c1 - c0);
        }
        const double cp = (r > 0.) ? x / r : 1.;
        const double sp = (r > 0.) ? y / r : 0.;
        out[0] = bc[0] * cp - bc[1] * sp;
        out[1] = bc[0] * sp + bc[1] * cp;
        out[2] = bc[2];
    }
};

}  // namespace oracle_field
