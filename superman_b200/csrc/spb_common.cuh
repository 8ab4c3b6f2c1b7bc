// Shared device helpers: double-double arithmetic, Gray-code helpers, status
// codes and the per-device context used by every permanent kernel family.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "superman_b200.h"

#define SPB_CUDA_TRY(expr)                                                     \
    do {                                                                       \
        cudaError_t _e = (expr);                                               \
        if (_e != cudaSuccess) {                                               \
            spb_set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                          __FILE__, __LINE__);                                 \
            return SPB_ERR_CUDA;                                               \
        }                                                                      \
    } while (0)

// Records a human-readable message for spb_last_error() (thread-local).
void spb_set_error(const char* fmt, ...);

namespace spb {

// ---------------------------------------------------------- double-double --
// Error-free transformations (Knuth TwoSum, Dekker Fast2Sum).  Written with
// explicit round-to-nearest intrinsics so the compiler cannot contract or
// reassociate them.
struct dd {
    double hi, lo;
};

__host__ __device__ __forceinline__ double add_rn(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    volatile double s = a + b;
    return s;
#endif
}
__host__ __device__ __forceinline__ double sub_rn(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    volatile double s = a - b;
    return s;
#endif
}
__host__ __device__ __forceinline__ double mul_rn(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    volatile double s = a * b;
    return s;
#endif
}

__host__ __device__ __forceinline__ dd two_sum(double a, double b)
{
    double s = add_rn(a, b);
    double bb = sub_rn(s, a);
    double e = add_rn(sub_rn(a, sub_rn(s, bb)), sub_rn(b, bb));
    return {s, e};
}

__host__ __device__ __forceinline__ dd fast_two_sum(double a, double b)
{
    double s = add_rn(a, b);
    double e = sub_rn(b, sub_rn(s, a));
    return {s, e};
}

__host__ __device__ __forceinline__ dd dd_add_d(dd a, double b)
{
    dd s = two_sum(a.hi, b);
    return fast_two_sum(s.hi, add_rn(s.lo, a.lo));
}

__host__ __device__ __forceinline__ dd dd_add(dd a, dd b)
{
    dd s = two_sum(a.hi, b.hi);
    dd t = two_sum(a.lo, b.lo);
    s = fast_two_sum(s.hi, add_rn(s.lo, t.hi));
    return fast_two_sum(s.hi, add_rn(s.lo, t.lo));
}

__host__ __device__ __forceinline__ dd dd_neg(dd a) { return {-a.hi, -a.lo}; }

// a + b left unnormalised: hi = fl(a.hi + b.hi), lo = its rounding error
// plus both lo words.  About 2^-106 (|a| + |b|) off; 8 operations against 20
// for dd_add, for a factor that goes straight into dd_mul (which takes an
// unnormalised operand and returns a normalised product).
__host__ __device__ __forceinline__ dd dd_add_fast(dd a, dd b)
{
    const dd s = two_sum(a.hi, b.hi);
    return {s.hi, add_rn(s.lo, add_rn(a.lo, b.lo))};
}

// (a.hi + a.lo) * (b.hi + b.lo) to ~2^-104 relative (Dekker product with FMA).
__device__ __forceinline__ dd dd_mul(dd a, dd b)
{
    double p = __dmul_rn(a.hi, b.hi);
    double e = __fma_rn(a.hi, b.hi, -p);
    e = __fma_rn(a.hi, b.lo, e);
    e = __fma_rn(a.lo, b.hi, e);
    return fast_two_sum(p, e);
}

// ---------------------------------------------------------------- shuffles --
__device__ __forceinline__ dd shfl_xor_dd(dd v, int lane_mask)
{
    return {__shfl_xor_sync(0xffffffffu, v.hi, lane_mask),
            __shfl_xor_sync(0xffffffffu, v.lo, lane_mask)};
}

__device__ __forceinline__ dd warp_sum_dd(dd v)
{
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v = dd_add(v, shfl_xor_dd(v, m));
    return v;
}

// ---------------------------------------------------------------- helpers --
__host__ __device__ __forceinline__ unsigned long long gray_of(unsigned long long k)
{
    return k ^ (k >> 1);
}

// Static, balanced split of [0, total) over `parts`: part t gets
// [t*base + min(t, rem), ...) with base = total / parts, rem = total % parts.
__host__ __device__ __forceinline__ void balanced_range(unsigned long long total,
                                                        unsigned long long parts,
                                                        unsigned long long t,
                                                        unsigned long long* begin,
                                                        unsigned long long* end)
{
    unsigned long long base = total / parts, rem = total % parts;
    unsigned long long b = t * base + (t < rem ? t : rem);
    *begin = b;
    *end = b + base + (t < rem ? 1ull : 0ull);
}

}  // namespace spb
