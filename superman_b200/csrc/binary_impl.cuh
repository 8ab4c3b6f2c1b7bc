// Exact 0/1 permanent by the Nijenhuis–Wilf form of Ryser's formula in
// integers.  With x'_r(S) = 2 a_{r,n-1} - rowsum_r + 2 sum_{j in S} a_rj
// (twice the NW row value, an integer in [-n, n]) over the subsets S of
// columns 0..n-2,
//   Sigma = sum_S (-1)^|S| prod_r x'_r(S) = 2^(n-1) * (+-) perm(A)
// (+ for odd n, - for even), computed in wrap-around integer arithmetic
// modulo 2^(32L).  The host picks L from a Bregman-Minc bound so that
// |Sigma| < 2^(32L-1), then shifts Sigma right by n-1 bits: the result is
// exact.  Half the subsets of plain Ryser, for n - 1 more accumulator bits.
//
// The reference has no integer path: 0/1 input goes through its FP64 NW
// walk (IO/IO.h:441-443 feeding Algorithms/GPU/Dense/dpSingleGPU.cuh), whose
// result is off by ~1e-10 relative at n=30.
//
// Layout mirrors the dense walk: the w low columns are enumerated from a
// shared table DEI[d][r] = twice the number of ones of row r among the
// columns of d (grouped [d/4][r][d%4], so one 16-byte broadcast load serves
// four terms); the n-1-w high columns form a unit index walked in Gray order
// per thread with the unit base xtop_r in registers.
//
// Each term's product is formed in two stages.  The row values and the
// products of K consecutive rows ("words") are small integers held in FP32,
// where they are exact: |x'_r| <= n and K is the largest count with
// n^K < 2^23, so every sum and product is an integer below 2^24.  A word's
// magnitude becomes an unsigned integer by adding 2^23 to |v| (exact in
// [2^23, 2^24), where the mantissa is |v| itself) and its sign bit is
// collected by xor.  The word magnitudes are then multiplied together in L
// 32-bit limbs with 32x32->64 multiply-adds, only over the limbs the bit
// widths so far can reach, and the term is added or subtracted once.  The
// row arithmetic thus runs on the FP32 pipe (twice the integer
// multiply-add rate) and the integer pipes keep only the limb work.  Unit
// sums and the grid reduction are exact, so the result does not depend on
// the launch shape.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "spb_common.cuh"

namespace spb {
namespace binary {

constexpr int kMaxN = 63;
constexpr int kMaxLimbs = 12;   // accumulator limbs (the result needs at most 10)

struct Problem {
    int n, w, limbs, grid;
    unsigned long long units;  // 2^(n-1-w) Gray units of 2^w terms each
    const float* x0;           // [n] 2 a_{r,n-1} - rowsum_r
    const float* dei;          // [2^w/4][n][4] twice the low-column row counts
    const float* mt;           // [n-1-w][n] high columns, doubled (0/2)
    uint32_t* partials;        // [grid][limbs]
    unsigned* ticket;          // last-CTA election (reset by the kernel)
    uint32_t* result;          // [limbs] sum over subsets, mod 2^(32*limbs)
};

// Rows per FP32 word: the largest K with n^K < 2^23 (|x'_r| <= n, so every
// partial product of a word is an integer the FP32 mantissa holds exactly,
// and |word| + 2^23 stays below 2^24).
__host__ __device__ constexpr int rows_per_word(int n)
{
    int k = 1;
    const unsigned long long b = (unsigned long long)(n > 1 ? n : 2);
    unsigned long long p = b;
    while (p * b < (1ull << 23) && k < 22) {
        p *= b;
        ++k;
    }
    return k;
}

// Bit width of n^k, the largest magnitude of a word of k rows.
__host__ __device__ constexpr int word_bits(int n, int k)
{
    unsigned long long p = 1;
    for (int i = 0; i < k; ++i) p *= (unsigned long long)n;
    int b = 0;
    while (b < 63 && (1ull << b) <= p) ++b;
    return b;
}

// Limbs that can be nonzero in the product of words 0..g (at most L).
__host__ __device__ constexpr int limbs_after(int n, int g, int L)
{
    const int K = rows_per_word(n);
    int bits = 0;
    for (int h = 0; h <= g; ++h) {
        const int rows = n - h * K < K ? n - h * K : K;
        bits += word_bits(n, rows);
    }
    const int l = (bits + 31) / 32;
    return l < L ? l : L;
}

// a += p, or a -= p when sub, modulo 2^(32L): a + (p xor mask) + sub.
template <int L>
__device__ __forceinline__ void limb_add_signed(uint32_t (&a)[L], const uint32_t (&p)[L], bool sub)
{
    const uint32_t mask = sub ? 0xffffffffu : 0u;
    uint64_t c = sub ? 1u : 0u;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        uint64_t t = (uint64_t)a[i] + (p[i] ^ mask) + c;
        a[i] = (uint32_t)t;
        c = t >> 32;
    }
}

// a += p when mask is 0, a -= p when mask is all ones, modulo 2^(32L).
template <int L>
__device__ __forceinline__ void limb_add_masked(uint32_t (&a)[L], const uint32_t (&p)[L], uint32_t mask)
{
    uint64_t c = mask & 1u;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        uint64_t t = (uint64_t)a[i] + (p[i] ^ mask) + c;
        a[i] = (uint32_t)t;
        c = t >> 32;
    }
}

template <int L>
__device__ __forceinline__ void limb_add(uint32_t (&a)[L], const uint32_t (&b)[L])
{
    uint64_t c = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        uint64_t t = (uint64_t)a[i] + b[i] + c;
        a[i] = (uint32_t)t;
        c = t >> 32;
    }
}

template <int L>
__device__ __forceinline__ void limb_sub(uint32_t (&a)[L], const uint32_t (&b)[L])
{
    uint64_t br = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        uint64_t t = (uint64_t)a[i] - b[i] - br;
        a[i] = (uint32_t)t;
        br = (t >> 63) & 1ull;
    }
}

// Sum over one unit: sum_d (-1)^popc(d) prod_r (xt_r + DEI[d][r]), the four
// terms of a group side by side (one 16-byte table load per row serves all
// four).  Per word: the FP32 product of its rows for each term, its sign bit
// xor-ed into the term's sign, its magnitude multiplied into the term's limbs.
template <int N, int L>
__device__ __forceinline__ void unit_sum_bin(const float (&xt)[N], const float* __restrict__ s_de, int nq,
                                             uint32_t (&acc)[L])
{
    constexpr int K = rows_per_word(N);
    constexpr int NG = (N + K - 1) / K;
#pragma unroll
    for (int l = 0; l < L; ++l) acc[l] = 0u;
#pragma unroll 1
    for (int q = 0; q < nq; ++q) {
        const float4* de = reinterpret_cast<const float4*>(s_de + q * (N * 4));
        uint32_t p[4][L];
        uint32_t sg[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int l = 0; l < L; ++l) p[i][l] = 0u;
#pragma unroll
        for (int g = 0; g < NG; ++g) {
            float v[4];
            {
                const int r = g * K;
                const float4 d = de[r];
                v[0] = __fadd_rn(xt[r], d.x);
                v[1] = __fadd_rn(xt[r], d.y);
                v[2] = __fadd_rn(xt[r], d.z);
                v[3] = __fadd_rn(xt[r], d.w);
            }
#pragma unroll
            for (int k = 1; k < K; ++k) {
                const int r = g * K + k;
                if (r < N) {
                    const float4 d = de[r];
                    v[0] = __fmul_rn(v[0], __fadd_rn(xt[r], d.x));
                    v[1] = __fmul_rn(v[1], __fadd_rn(xt[r], d.y));
                    v[2] = __fmul_rn(v[2], __fadd_rn(xt[r], d.z));
                    v[3] = __fmul_rn(v[3], __fadd_rn(xt[r], d.w));
                }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                sg[i] ^= __float_as_uint(v[i]);
                const uint32_t m = __float_as_uint(__fadd_rn(fabsf(v[i]), 8388608.0f)) - 0x4B000000u;
                if (g == 0) {
                    p[i][0] = m;
                } else {
                    // p *= m over the limbs words 0..g-1 can reach; the carry
                    // out lands in the next limb (dropped past L: mod 2^(32L))
                    const int nb = limbs_after(N, g - 1, L);
                    uint64_t c = 0;
#pragma unroll
                    for (int l = 0; l < L; ++l)
                        if (l < nb) {
                            const uint64_t t = (uint64_t)p[i][l] * m + c;
                            p[i][l] = (uint32_t)t;
                            c = t >> 32;
                        }
#pragma unroll
                    for (int l = 0; l < L; ++l)
                        if (l == nb) p[i][l] = (uint32_t)c;
                }
            }
        }
        // signs: the product's (bit 31 of sg) and the group pattern + - - +
        // relative to popc(q); an all-ones mask subtracts
        const uint32_t flip = (__popc(q) & 1) ? 0x80000000u : 0u;
        limb_add_masked<L>(acc, p[0], (uint32_t)((int32_t)(sg[0] ^ flip) >> 31));
        limb_add_masked<L>(acc, p[1], (uint32_t)((int32_t)(sg[1] ^ flip ^ 0x80000000u) >> 31));
        limb_add_masked<L>(acc, p[2], (uint32_t)((int32_t)(sg[2] ^ flip ^ 0x80000000u) >> 31));
        limb_add_masked<L>(acc, p[3], (uint32_t)((int32_t)(sg[3] ^ flip) >> 31));
    }
}

template <int L>
__device__ __forceinline__ void shfl_add(uint32_t (&v)[L], int m)
{
    uint32_t o[L];
#pragma unroll
    for (int l = 0; l < L; ++l) o[l] = __shfl_xor_sync(0xffffffffu, v[l], m);
    limb_add<L>(v, o);
}

// Threads per CTA: 512 (128 registers) keeps 4 limbs spill-free up to
// n = 28 except n = 27 (seven words, the last of three rows); larger n or
// more limbs get 255 registers at 256 threads.
__host__ __device__ constexpr int bin_max_threads(int n, int limbs)
{
    return (limbs <= 4 && n <= 28 && n != 27) ? 512 : 256;
}

template <int N, int L>
__global__ void __launch_bounds__(bin_max_threads(N, L), 1) walk_binary(Problem pb)
{
    constexpr int G = 4;
    extern __shared__ __align__(16) float smem_f[];
    const int w = pb.w, terms = 1 << w, nq = terms / G, ntop = N - 1 - w;
    const int tid = threadIdx.x, bd = blockDim.x;
    float* s_de = smem_f;
    float* s_mt = s_de + terms * N;
    for (int i = tid; i < terms * N; i += bd) s_de[i] = pb.dei[i];
    for (int i = tid; i < ntop * N; i += bd) s_mt[i] = pb.mt[i];
    __syncthreads();

    const unsigned long long T = (unsigned long long)gridDim.x * bd;
    const unsigned long long t = (unsigned long long)blockIdx.x * bd + tid;
    unsigned long long u0, u1;
    balanced_range(pb.units, T, t, &u0, &u1);
    uint32_t tot[L];
#pragma unroll
    for (int l = 0; l < L; ++l) tot[l] = 0u;
    if (u0 < u1) {
        float xt[N];  // small integers, exact in FP32
        const unsigned long long g0 = gray_of(u0);
#pragma unroll
        for (int r = 0; r < N; ++r) xt[r] = pb.x0[r];
        for (int j = 0; j < ntop; ++j) {  // columns outermost, rows independent
            if (!((g0 >> j) & 1ull)) continue;
#pragma unroll
            for (int r = 0; r < N; ++r) xt[r] = __fadd_rn(xt[r], s_mt[j * N + r]);
        }
        unsigned long long u = u0;
        while (true) {
            uint32_t us[L];
            unit_sum_bin<N, L>(xt, s_de, nq, us);
            if (u & 1ull) limb_sub<L>(tot, us);
            else limb_add<L>(tot, us);
            if (++u >= u1) break;
            const int j = __ffsll((long long)u) - 1;
            const bool add = (gray_of(u) >> j) & 1ull;
            const float* col = s_mt + j * N;
#pragma unroll
            for (int r = 0; r < N; ++r) xt[r] = add ? __fadd_rn(xt[r], col[r]) : __fsub_rn(xt[r], col[r]);
        }
    }
    // warp -> block -> grid (exact; order only affects speed)
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) shfl_add<L>(tot, m);
    __shared__ uint32_t s_warp[16][kMaxLimbs];
    __shared__ int s_last;
    const int lane = tid & 31, wid = tid >> 5, nw = bd >> 5;
    if (lane == 0)
#pragma unroll
        for (int l = 0; l < L; ++l) s_warp[wid][l] = tot[l];
    __syncthreads();
    if (wid == 0) {
        uint32_t v[L];
#pragma unroll
        for (int l = 0; l < L; ++l) v[l] = lane < nw ? s_warp[lane][l] : 0u;
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) shfl_add<L>(v, m);
        if (lane == 0) {
#pragma unroll
            for (int l = 0; l < L; ++l) pb.partials[blockIdx.x * L + l] = v[l];
            __threadfence();
            unsigned prev = atomicAdd(pb.ticket, 1u);
            s_last = (prev == gridDim.x - 1) ? 1 : 0;
        }
    }
    __syncthreads();
    if (s_last && wid == 0) {
        __threadfence();
        uint32_t v[L];
#pragma unroll
        for (int l = 0; l < L; ++l) v[l] = 0u;
        for (int b = lane; b < (int)gridDim.x; b += 32) {
            uint32_t o[L];
#pragma unroll
            for (int l = 0; l < L; ++l) o[l] = __ldcg(pb.partials + b * L + l);
            limb_add<L>(v, o);
        }
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) shfl_add<L>(v, m);
        if (lane == 0) {
#pragma unroll
            for (int l = 0; l < L; ++l) pb.result[l] = v[l];
            *pb.ticket = 0u;
        }
    }
}

int launch_binary(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s);

}  // namespace binary
}  // namespace spb
