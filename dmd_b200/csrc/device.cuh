// device.cuh -- device helpers shared by the kernel translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "layout.h"

namespace dmd {

constexpr unsigned FULL = 0xffffffffu;

// Cell::minimum_image, orthorhombic branch (src/core/cell.cpp:26-38), with the
// reference's rounding: d - round(d * (1/L)) * L, no contraction.  CUDA's
// round() rounds half away from zero like std::round.
__device__ __forceinline__ double mi_ref(double d, double L, double invL) {
    return __dsub_rn(d, __dmul_rn(round(__dmul_rn(d, invL)), L));
}

// dx*dx + dy*dy + dz*dz evaluated left to right without FMA.
__device__ __forceinline__ double r2_ref(double dx, double dy, double dz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ __forceinline__ void set_status(RepState* s, int flag) { atomicOr(&s->status, flag); }

// Fixed-point conversion with range / NaN detection (the value is clamped so the
// integer conversion is always defined).
template <typename T>
__device__ __forceinline__ long long to_fix(T v, double scale, RepState* s) {
    double d = static_cast<double>(v);
    if (!(fabs(d) < FMAX)) {
        set_status(s, (d != d) ? ST_NAN : ST_RANGE);
        d = (d != d) ? 0.0 : copysign(FMAX, d);
    }
    return __double2ll_rn(d * scale);
}

__device__ __forceinline__ void fix_add(long long* p, long long v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

__device__ __forceinline__ double from_fix(long long v, double scale) {
    return static_cast<double>(v) * (1.0 / scale);
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ double warp_min_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

// Replica of a flat chunk number (chunk_prefix has n_rep + 1 entries).
__device__ __forceinline__ int chunk_replica(const int* prefix, int n_rep, int w) {
    int lo = 0, hi = n_rep;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (prefix[mid] <= w) lo = mid; else hi = mid;
    }
    return lo;
}

// CoulombPME::theta4 / dtheta4 (src/force/coulomb_pme.cpp:50-69)
template <typename T>
__device__ __forceinline__ T theta4(T u) {
    T a = fabs(u);
    if (a >= T(2)) return T(0);
    if (a >= T(1)) {
        T t = T(2) - a;
        return t * t * t / T(6);
    }
    return (T(4) - T(6) * a * a + T(3) * a * a * a) / T(6);
}

template <typename T>
__device__ __forceinline__ T dtheta4(T u) {
    T a = fabs(u);
    if (a >= T(2)) return T(0);
    T s = (u >= T(0)) ? T(1) : T(-1);
    if (a >= T(1)) {
        T t = T(2) - a;
        return -s * t * t / T(2);
    }
    return s * (T(9) * a * a - T(12) * a) / T(6);
}

}  // namespace dmd
