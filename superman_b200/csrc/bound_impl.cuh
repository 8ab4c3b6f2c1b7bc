// Bound-only pre-pass of the double-double mode: counts the Gray units per
// bound bin before the first walk, so that the walk can list every unit in
// the top bins as it goes (dense_impl.cuh, raw_list_add).
//
// Only the counts near the top of the distribution matter, and only to choose
// the listing bin, so the pass runs in FP32 with x_r in registers.  The
// bound U = prod_r f_r, f_r = max_d |x_r + DE[d][r]|, is a product of row
// factors clamped to [2^-24, 2^24] whose exponent is moved into an integer
// every 4 rows (so the product never leaves the float range); for real rows
// f_r = |x_r + mid_r| + half_r with mid/half the centre and half-width of the
// row's DE range, so the walk keeps y_r = x_r + mid_r.  Near a bin edge the
// bin may differ from the walk's FP64 bin; that shifts the list length,
// never the result.
#pragma once

#include "dense_impl.cuh"

namespace spb {
namespace dense {

// Column stride of the high columns in shared memory: a multiple of 4 floats
// (16-byte rows, so row runs load as 16-byte vectors) whose quarter is odd,
// so that lanes reading different columns j (each thread steps its own Gray
// unit) at the same row fall in different 16-byte bank groups for j mod 8.
__host__ __device__ constexpr int bound_col_stride(int n)
{
    return (((n + 3) & ~3) >> 2) & 1 ? ((n + 3) & ~3) : ((n + 3) & ~3) + 4;
}

// Shared memory: high columns and bound terms as floats, then the counts.
__host__ __device__ inline size_t bound_smem_bytes_f(int n, int c, int w)
{
    const int ntp = n - 1 - w > 0 ? n - 1 - w : 0;
    return sizeof(float) * ((size_t)c * ntp * bound_col_stride(n) + 2 * n) + sizeof(unsigned) * kHistBins;
}

// Moves the binary exponent of p (normal, positive) into e; p keeps [1, 2).
__device__ __forceinline__ void bound_renorm(float& p, int& e)
{
    const int bits = __float_as_int(p);
    e += ((bits >> 23) & 0xff) - 127;
    p = __int_as_float((bits & 0x007fffff) | 0x3f800000);
}

template <int N, int C>
__global__ void __launch_bounds__(256) bound_walk(Problem pb)
{
    extern __shared__ __align__(16) float fsm[];
    constexpr int S = bound_col_stride(N);
    const int ntop = N - 1 - pb.w, ntp = ntop > 0 ? ntop : 0;
    const int tid = threadIdx.x, bd = blockDim.x, lane = tid & 31;
    float* s_mt = fsm;                   // [C][ntop][S], rows 0..N-1 used
    float* s_b = s_mt + C * ntp * S;     // real [2][N] (mid, half), complex [N] (max |DE|)
    unsigned* s_cnt = reinterpret_cast<unsigned*>(s_b + 2 * N);
    for (int i = tid; i < C * ntp * N; i += bd) s_mt[(i / N) * S + i % N] = (float)pb.mt[i];
    for (int r = tid; r < N; r += bd) {
        if constexpr (C == 1) {
            s_b[r] = (float)(0.5 * (pb.bnd[r] + pb.bnd[N + r]));
            s_b[N + r] = (float)(0.5 * (pb.bnd[N + r] - pb.bnd[r]));
        } else {
            s_b[r] = (float)pb.bnd[r];
        }
    }
    for (int i = tid; i < kHistBins; i += bd) s_cnt[i] = 0u;
    __syncthreads();

    const unsigned long long T = (unsigned long long)gridDim.x * bd;
    const unsigned long long t = (unsigned long long)blockIdx.x * bd + tid;
    unsigned long long u0, u1;
    balanced_range(pb.units, T, t, &u0, &u1);
    float x[C][N], hb[N];
    const unsigned long long g0 = gray_of(u0);
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
        for (int r = 0; r < N; ++r) x[c][r] = (float)pb.x0_hi[c * N + r] + (C == 1 ? s_b[r] : 0.0f);  // real: y = x + mid
    for (int j = 0; j < ntop; ++j) {  // columns outermost, rows independent
        if (!((g0 >> j) & 1ull)) continue;
#pragma unroll
        for (int c = 0; c < C; ++c)
#pragma unroll
            for (int r = 0; r < N; ++r) x[c][r] += s_mt[(c * ntp + j) * S + r];
    }
#pragma unroll
    for (int r = 0; r < N; ++r) hb[r] = C == 1 ? s_b[N + r] : s_b[r];
    for (unsigned long long u = u0; u < u1; ++u) {
        if (u > u0) {
            const int j = __ffsll((long long)u) - 1;
            const float sg = ((gray_of(u) >> j) & 1ull) ? 1.0f : -1.0f;
#pragma unroll
            for (int c = 0; c < C; ++c)
#pragma unroll
                for (int r = 0; r < N; ++r) x[c][r] = fmaf(sg, s_mt[(c * ntp + j) * S + r], x[c][r]);
        }
        float p = 1.0f;
        int e = 0;
#pragma unroll
        for (int r = 0; r < N; ++r) {
            float f;
            if constexpr (C == 1) f = fabsf(x[0][r]) + hb[r];
            else {
                const float m2 = fmaxf(fmaf(x[0][r], x[0][r], x[C - 1][r] * x[C - 1][r]), 0x1p-100f);
                f = m2 * rsqrtf(m2) + hb[r];  // |x| to a few ulps: an estimate
            }
            p *= fminf(fmaxf(f, 0x1p-24f), 0x1p24f);
            if ((r & 3) == 3) bound_renorm(p, e);
        }
        bound_renorm(p, e);
        int b = (e + 1024) >> 2;  // e = floor(log2 U), as ilogb in hist_bin
        b = b < 0 ? 0 : (b >= kHistBins ? kHistBins - 1 : b);
        const unsigned same = __match_any_sync(__activemask(), b);
        if (lane == __ffs(same) - 1) atomicAdd(&s_cnt[b], (unsigned)__popc(same));
    }
    __syncthreads();
    for (int i = tid; i < kHistBins; i += bd)
        if (s_cnt[i]) atomicAdd(&pb.pre_cnt[i], s_cnt[i]);
}

}  // namespace dense
}  // namespace spb
