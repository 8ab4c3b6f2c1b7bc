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
// per thread with the integer unit base xtop_r in registers.  Each term
// multiplies its row values in words of up to K rows (n^K < 2^32: the word's
// magnitude is an exact unsigned 32-bit integer), folds the word magnitudes
// into L 32-bit limbs with 32x32->64 multiply-adds over only the limbs the
// bit widths so far can reach, and applies the sign (the xor of the words')
// once.  Unit sums and the grid reduction are exact, so the result does not
// depend on the launch shape.
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
    const int* x0;             // [n] 2 a_{r,n-1} - rowsum_r
    const int* dei;            // [2^w/4][n][4] twice the low-column row counts
    const int8_t* mt;          // [n-1-w][n] high columns, doubled (0/2)
    uint32_t* partials;        // [grid][limbs]
    unsigned* ticket;          // last-CTA election (reset by the kernel)
    uint32_t* result;          // [limbs] sum over subsets, mod 2^(32*limbs)
};

// Rows per word: the largest K with n^K < 2^32, so a word's magnitude fits
// an unsigned 32-bit integer (|x'_r| <= n).  Its first K-1 rows multiply in
// signed 32-bit arithmetic (n^(K-1) < 2^31: exact); the last row's magnitude
// multiplies the magnitude of that product, unsigned.
__host__ __device__ constexpr int rows_per_word(int n)
{
    int k = 1;
    const unsigned long long b = (unsigned long long)(n > 1 ? n : 2);
    unsigned long long p = b;
    while (p * b < (1ull << 32) && k < 16) {
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

// Limbs that can be nonzero in the product of words 0..g (at most L): the
// bit widths of the words so far, summed, in 32-bit limbs.
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

// Word g of a term (rows g*K .. g*K + rows - 1): the signed product of its
// first rows, then the unsigned product of the magnitudes with its last row;
// its sign bit is xor-ed into sg and its magnitude multiplied into the limbs
// that the bit widths of words 0..g-1 can reach (a compile-time count), the
// carry out of the top one landing in the next (dropped past L: mod 2^(32L)).
// Recurses over g so that every count is a constant.
template <int N, int L, int G, int g>
__device__ __forceinline__ void term_word(const int (&xt)[N], const int* __restrict__ de, int i,
                                          uint32_t (&p)[L], uint32_t& sg)
{
    constexpr int K = rows_per_word(N);
    constexpr int NG = (N + K - 1) / K;
    constexpr int r0 = g * K, rows = N - r0 < K ? N - r0 : K;
    uint32_t m;
    if constexpr (rows == 1) {
        const int x = xt[r0] + de[r0 * G + i];
        sg ^= (uint32_t)x;
        m = (uint32_t)(x < 0 ? -x : x);
    } else {
        int sw = xt[r0] + de[r0 * G + i];
#pragma unroll
        for (int k = 1; k < rows - 1; ++k) sw *= xt[r0 + k] + de[(r0 + k) * G + i];
        const int x = xt[r0 + rows - 1] + de[(r0 + rows - 1) * G + i];
        sg ^= (uint32_t)sw ^ (uint32_t)x;
        m = (uint32_t)(sw < 0 ? -sw : sw) * (uint32_t)(x < 0 ? -x : x);
    }
    if constexpr (g == 0) {
        p[0] = m;
    } else {
        constexpr int nb = limbs_after(N, g - 1, L);
        uint64_t c = 0;
#pragma unroll
        for (int l = 0; l < nb; ++l) {
            const uint64_t t = (uint64_t)p[l] * m + c;
            p[l] = (uint32_t)t;
            c = t >> 32;
        }
        if constexpr (nb < L) p[nb] = (uint32_t)c;
    }
    if constexpr (g + 1 < NG) term_word<N, L, G, g + 1>(xt, de, i, p, sg);
}

// |prod_r x'_r| mod 2^(32L) for one term (x'_r = xt[r] + de(r), signed) into
// p; returns a word whose bit 31 is the product's sign (the xor of the
// factors' signs).
template <int N, int L, int G>
__device__ __forceinline__ uint32_t term_product(const int (&xt)[N], const int* __restrict__ de, int i,
                                                 uint32_t (&p)[L])
{
#pragma unroll
    for (int l = 0; l < L; ++l) p[l] = 0u;
    uint32_t sg = 0u;
    term_word<N, L, G, 0>(xt, de, i, p, sg);
    return sg;
}

// a += p when mask is 0, a -= p when mask is all ones, modulo 2^(32L).
template <int L>
__device__ __forceinline__ void limb_add_masked(uint32_t (&a)[L], const uint32_t (&p)[L], uint32_t mask)
{
    uint64_t c = mask & 1u;
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const uint64_t t = (uint64_t)a[l] + (p[l] ^ mask) + c;
        a[l] = (uint32_t)t;
        c = t >> 32;
    }
}

// Sum over one unit: sum_d (-1)^popc(d) prod_r (xt_r + DEI[d][r]).
template <int N, int L>
__device__ __forceinline__ void unit_sum_bin(const int (&xt)[N], const int* __restrict__ s_de, int nq,
                                             uint32_t (&acc)[L])
{
    constexpr int G = 4;
#pragma unroll
    for (int l = 0; l < L; ++l) acc[l] = 0u;
#pragma unroll 1
    for (int q = 0; q < nq; ++q) {
        const int* de = s_de + q * (N * G);
        // signs: the product's (bit 31 of the returned word) and the group
        // pattern + - - + relative to popc(q); an all-ones mask subtracts
        const uint32_t flip = (__popc(q) & 1) ? 0x80000000u : 0u;
        uint32_t p[L];
        uint32_t sg = term_product<N, L, G>(xt, de, 0, p);
        limb_add_masked<L>(acc, p, (uint32_t)((int32_t)(sg ^ flip) >> 31));
        sg = term_product<N, L, G>(xt, de, 1, p);
        limb_add_masked<L>(acc, p, (uint32_t)((int32_t)(sg ^ flip ^ 0x80000000u) >> 31));
        sg = term_product<N, L, G>(xt, de, 2, p);
        limb_add_masked<L>(acc, p, (uint32_t)((int32_t)(sg ^ flip ^ 0x80000000u) >> 31));
        sg = term_product<N, L, G>(xt, de, 3, p);
        limb_add_masked<L>(acc, p, (uint32_t)((int32_t)(sg ^ flip) >> 31));
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
// n = 28; larger n or more limbs get 255 registers at 256 threads.
__host__ __device__ constexpr int bin_max_threads(int n, int limbs) { return (limbs <= 4 && n <= 28) ? 512 : 256; }

template <int N, int L>
__global__ void __launch_bounds__(bin_max_threads(N, L), 1) walk_binary(Problem pb)
{
    constexpr int G = 4;
    extern __shared__ __align__(16) int smem_i[];
    const int w = pb.w, terms = 1 << w, nq = terms / G, ntop = N - 1 - w;
    const int tid = threadIdx.x, bd = blockDim.x;
    int* s_de = smem_i;
    int8_t* s_mt = reinterpret_cast<int8_t*>(s_de + terms * N);
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
        int xt[N];
        const unsigned long long g0 = gray_of(u0);
#pragma unroll
        for (int r = 0; r < N; ++r) xt[r] = pb.x0[r];
        for (int j = 0; j < ntop; ++j) {  // columns outermost, rows independent
            if (!((g0 >> j) & 1ull)) continue;
#pragma unroll
            for (int r = 0; r < N; ++r) xt[r] += s_mt[j * N + r];
        }
        unsigned long long u = u0;
        while (true) {
            uint32_t us[L];
            unit_sum_bin<N, L>(xt, s_de, nq, us);
            if (u & 1ull) limb_sub<L>(tot, us);
            else limb_add<L>(tot, us);
            if (++u >= u1) break;
            const int j = __ffsll((long long)u) - 1;
            const int sg = ((gray_of(u) >> j) & 1ull) ? 1 : -1;
            const int8_t* col = s_mt + j * N;
#pragma unroll
            for (int r = 0; r < N; ++r) xt[r] += sg * col[r];
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

// Launches walk_binary<pb.n, pb.limbs>; with per_sm set, launches nothing
// and stores the CTAs per SM that the launch shape allows.
int launch_binary(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s, int* per_sm = nullptr);

}  // namespace binary
}  // namespace spb
