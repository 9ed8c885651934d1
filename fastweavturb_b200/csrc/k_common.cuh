// k_common.cuh -- device helpers shared by the kernels of libfwt.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "fwt_internal.h"

namespace fwt {

__device__ __forceinline__ double dev_pi() { return 3.141592653589793115997963468544185161590576171875; }
__device__ __forceinline__ double dev_pi2() { return 6.28318530717958623199592693708837032318115234375; }

// Exact FP64 arithmetic steps (no FMA contraction) for the statements that decide integer
// outcomes (box bounds, sub-segment counts), so they follow the reference's rounding.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// cuFFT's complex type of a real precision
template <typename Real>
struct Cplx;
template <>
struct Cplx<float> {
    using T = cufftComplex;
};
template <>
struct Cplx<double> {
    using T = cufftDoubleComplex;
};

// Quintic spline evaluation (subroutine.f90:490-560); coe layout [coord][6].
__device__ __forceinline__ void spl_pos(const double *coe, double z, double *c3)
{
    const double z2 = dmul(z, z), z3 = dmul(z2, z), z4 = dmul(z3, z), z5 = dmul(z4, z);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double *a = coe + 6 * d;
        double v = dmul(a[5], z5);
        v = dadd(v, dmul(a[4], z4));
        v = dadd(v, dmul(a[3], z3));
        v = dadd(v, dmul(a[2], z2));
        v = dadd(v, dmul(a[1], z));
        v = dadd(v, a[0]);
        if (v >= dev_pi()) v = dsub(v, dev_pi2());
        if (v < -dev_pi()) v = dadd(v, dev_pi2());
        c3[d] = v;
    }
}

__device__ __forceinline__ void spl_d1(const double *coe, double z, double *c3)
{
    const double z2 = dmul(z, z), z3 = dmul(z2, z), z4 = dmul(z3, z);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double *a = coe + 6 * d;
        double v = dmul(dmul(5.0, a[5]), z4);
        v = dadd(v, dmul(dmul(4.0, a[4]), z3));
        v = dadd(v, dmul(dmul(3.0, a[3]), z2));
        v = dadd(v, dmul(dmul(2.0, a[2]), z));
        v = dadd(v, a[1]);
        c3[d] = v;
    }
}

__device__ __forceinline__ void spl_d2(const double *coe, double z, double *c3)
{
    const double z2 = dmul(z, z), z3 = dmul(z2, z);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double *a = coe + 6 * d;
        double v = dmul(dmul(20.0, a[5]), z3);
        v = dadd(v, dmul(dmul(12.0, a[4]), z2));
        v = dadd(v, dmul(dmul(6.0, a[3]), z));
        v = dadd(v, dmul(2.0, a[2]));
        c3[d] = v;
    }
}

__device__ __forceinline__ double sigma_func(double zeta, double length, double smax, double smin, int n_T)
{
    // subroutine.f90:164-173; a constant core gives smin + 0 * (...) = smin exactly
    if (smax == smin) return smin;
    const double omega = floor(length / dev_pi() + 0.5) * (double)n_T;
    return smin + (smax - smin) * (sin(omega * zeta) + 1.0) / 2.0;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// positive modulo for wrapping unwrapped grid indices
__device__ __forceinline__ int wrap_idx(int i, int n)
{
    int r = i % n;
    return r < 0 ? r + n : r;
}

// float <-> order-preserving uint32 (for bit-exact atomic min/max)
__device__ __forceinline__ uint32_t f2ord(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float ord2f(uint32_t u)
{
    uint32_t v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(v);
#else
    float f;
    __builtin_memcpy(&f, &v, 4);
    return f;
#endif
}

// double <-> order-preserving uint64 (bit-exact atomic min/max of FP64 values)
__device__ __forceinline__ unsigned long long d2ord(double f)
{
    const unsigned long long u = (unsigned long long)__double_as_longlong(f);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ double ord2d(unsigned long long u)
{
    const unsigned long long v = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)v);
#else
    double f;
    __builtin_memcpy(&f, &v, 8);
    return f;
#endif
}

}  // namespace fwt
