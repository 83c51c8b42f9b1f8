// Basic definitions shared by every device module of the propagator.
//
// All hot-path code is written once as templates over the scalar type S
// (float on the production path, double for the fp64 build) and compiled for
// sm_100a.  Functions are marked DPROP_HD so that the same source also builds
// with a host compiler for unit-level checks; the library itself only ever
// runs them on the device.
#pragma once

#include <stdint.h>

#include <cfloat>
#include <cmath>

#if !defined(__CUDACC__)
#include <vector_types.h>  // float4 for the host build of the core
#endif

#if defined(__CUDACC__)
#define DPROP_HD __host__ __device__ __forceinline__
#define DPROP_D __device__ __forceinline__
// Infrequently taken paths (volume re-initialisation, covariance transport,
// material).  Inlined by default: measured on B200, keeping them out of line
// forces the track state into the stack frame and costs more than the
// instruction-cache locality it buys.  -DDPROP_OUTLINE_COLD keeps them out
// of line.
#if defined(DPROP_OUTLINE_COLD)
#define DPROP_HD_COLD __host__ __device__ __noinline__
#else
#define DPROP_HD_COLD __host__ __device__ __forceinline__
#endif
// Leaf functions with small interfaces (one surface intersection + mask
// check) that are called from several places; -DDPROP_OUTLINE_LEAF keeps a
// single out-of-line copy of each to shrink the kernel's code footprint.
#if defined(DPROP_OUTLINE_LEAF)
#define DPROP_HD_LEAF __host__ __device__ __noinline__
#else
#define DPROP_HD_LEAF __host__ __device__ __forceinline__
#endif
// Code only line (wire) surfaces and material rods reach: kept out of line
// so that detectors without them do not carry it in their hot loop
// (measured on B200: inlined, it slowed the toy detector's propagation by
// 11-14 %).
#define DPROP_HD_LINE __host__ __device__ __noinline__
#else
#define DPROP_HD_LINE inline
#define DPROP_HD inline
#define DPROP_D inline
#define DPROP_HD_COLD inline
#define DPROP_HD_LEAF inline
#endif

namespace dprop {

#if !defined(__CUDACC__)
using std::atan2;
using std::copysign;
using std::cos;
using std::fabs;
using std::floor;
using std::fma;
using std::isfinite;
using std::log;
using std::log10;
using std::pow;
using std::signbit;
using std::sin;
using std::sqrt;
#endif

// detray's internal units: mm, GeV, e; 1 T = 0.000299792458 GeV/(e mm)
// (core/include/detray/definitions/units.hpp:20-110).
namespace unit {
constexpr double um = 1e-3;
constexpr double mm = 1.0;
constexpr double MeV = 1e-3;
constexpr double eV = 1e-9;
constexpr double cm2 = 1e2;
constexpr double T = 0.000299792458;
}  // namespace unit

namespace constant {
constexpr double pi = 3.14159265358979323846;
constexpr double ln2 = 0.693147180559945309417;
constexpr double ln10 = 2.30258509299404568402;
constexpr double inv_sqrt2 = 0.70710678118654752440;
constexpr double m_e = 0.51099895069 * unit::MeV;
}  // namespace constant

template <typename S>
struct limits;
template <>
struct limits<float> {
    DPROP_HD static constexpr float max() { return FLT_MAX; }
    DPROP_HD static constexpr float epsilon() { return FLT_EPSILON; }
};
template <>
struct limits<double> {
    DPROP_HD static constexpr double max() { return DBL_MAX; }
    DPROP_HD static constexpr double epsilon() { return DBL_EPSILON; }
};

// ------------------------------------------------------------ 3-vectors
template <typename S>
struct vec3 {
    S x, y, z;
    DPROP_HD S operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

template <typename S>
DPROP_HD vec3<S> make3(S a, S b, S c) {
    return vec3<S>{a, b, c};
}
template <typename S>
DPROP_HD vec3<S> operator+(vec3<S> a, vec3<S> b) {
    return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <typename S>
DPROP_HD vec3<S> operator-(vec3<S> a, vec3<S> b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename S>
DPROP_HD vec3<S> operator*(S s, vec3<S> a) {
    return {s * a.x, s * a.y, s * a.z};
}
template <typename S>
DPROP_HD vec3<S> operator*(vec3<S> a, S s) {
    return {s * a.x, s * a.y, s * a.z};
}
template <typename S>
DPROP_HD S dot(vec3<S> a, vec3<S> b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename S>
DPROP_HD vec3<S> cross(vec3<S> a, vec3<S> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z,
            a.x * b.y - a.y * b.x};
}
template <typename S>
DPROP_HD S norm(vec3<S> a) {
    return sqrt(dot(a, a));
}
template <typename S>
DPROP_HD vec3<S> normalize(vec3<S> a) {
    return a * (S(1) / norm(a));
}
template <typename S>
DPROP_HD S perp(vec3<S> a) {
    return sqrt(fma(a.x, a.x, a.y * a.y));
}
template <typename S>
DPROP_HD S phi_of(vec3<S> a) {
    return atan2(a.y, a.x);
}
template <typename S>
DPROP_HD S theta_of(vec3<S> a) {
    return atan2(perp(a), a.z);
}

template <typename S>
DPROP_HD S min_(S a, S b) {
    return a < b ? a : b;
}
template <typename S>
DPROP_HD S max_(S a, S b) {
    return a > b ? a : b;
}

// ------------------------------------------------------- small matrices
// Row-major fixed-size matrix, used for the 3x3 blocks of the RK Jacobian.
template <typename S>
struct mat33 {
    S m[9];  // m[r * 3 + c]
    DPROP_HD S operator()(int r, int c) const { return m[r * 3 + c]; }
    DPROP_HD S& operator()(int r, int c) { return m[r * 3 + c]; }
};

template <typename S>
DPROP_HD mat33<S> identity33() {
    mat33<S> r{};
    for (int i = 0; i < 9; ++i) {
        r.m[i] = S(0);
    }
    r.m[0] = r.m[4] = r.m[8] = S(1);
    return r;
}

// Column-wise cross product: column j of the result is col_j(A) x v.
template <typename S>
DPROP_HD mat33<S> colwise_cross(const mat33<S>& a, vec3<S> v) {
    mat33<S> r;
    for (int j = 0; j < 3; ++j) {
        const vec3<S> c{a(0, j), a(1, j), a(2, j)};
        const vec3<S> x = cross(c, v);
        r(0, j) = x.x;
        r(1, j) = x.y;
        r(2, j) = x.z;
    }
    return r;
}

}  // namespace dprop
