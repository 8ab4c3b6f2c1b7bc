// Device helpers of the double-double refinement shared by its kernels
// (dense_refine.cu) and the fused small-matrix call (small_call.cu).
#pragma once

#include "dense_impl.cuh"

namespace spb {
namespace dense {

// One group of G terms, bitwise identical to unit_sum_real<N,G>'s group
// (na == n) or to unit_sum_sparse<NA>'s (na < n: the inactive rows' product
// first, then the na active rows; see sparse_impl.cuh).  The group's term i
// of row r is de[r * rs + i].
__device__ __forceinline__ double group_sum_real_rt(const double* xh, const double* de, int n, int na, int G,
                                                    int rs)
{
    double p0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
    p0 = add_rn(xh[0], de[0]);
    if (G >= 2) p1 = add_rn(xh[0], de[1]);
    if (G == 4) {
        p2 = add_rn(xh[0], de[2]);
        p3 = add_rn(xh[0], de[3]);
    }
    if (na < n) {
        double c = xh[na];
        for (int r = na + 1; r < n; ++r) c = mul_rn(c, xh[r]);
        p0 = mul_rn(c, p0);
        p1 = mul_rn(c, p1);
        p2 = mul_rn(c, p2);
        p3 = mul_rn(c, p3);
    }
    for (int r = 1; r < na; ++r) {
        const double x = xh[r];
        p0 = mul_rn(p0, add_rn(x, de[r * rs + 0]));
        if (G >= 2) p1 = mul_rn(p1, add_rn(x, de[r * rs + 1]));
        if (G == 4) {
            p2 = mul_rn(p2, add_rn(x, de[r * rs + 2]));
            p3 = mul_rn(p3, add_rn(x, de[r * rs + 3]));
        }
    }
    if (G == 4) return sub_rn(sub_rn(p0, p1), sub_rn(p2, p3));
    if (G == 2) return sub_rn(p0, p1);
    return p0;
}

// The refinement bin: the lowest bin b such that the units below it, left in
// FP64, have an expected rounding error sqrt(sum t^2 * k/12) * 2^-52 (k rounded
// operations per term) within half the tolerance of the walk's magnitude
// `mag`.  At most 1/8 of the units are refined; past that b moves up and the
// estimate is reported instead.  Called by all 32 lanes of one warp; lane l
// owns bins [16l, 16l + 16), and the cumulative sums over bins are lane-local
// sums joined by warp scans (a fixed order, so the result is deterministic).
// The histogram is read from a copy in shared memory laid out by
// hist_pad_index (staged with coalesced loads through L2: it was written by
// atomics of other CTAs).  Every lane returns the result.
struct ThresholdPick {
    int thr;                   // refinement bin (kHistBins: none)
    unsigned long long count;  // units at or above it
    double err;                // expected relative error of the units below it
};

// Shared-memory position of bin b in a staged copy of the histogram: each
// lane's 16 consecutive bins are one row of 17, so the lanes' reads of their
// i-th bins fall in different banks (two lanes per bank pair).
__host__ __device__ constexpr int hist_pad_index(int b)
{
    return (b / (kHistBins / 32)) * (kHistBins / 32 + 1) + b % (kHistBins / 32);
}
constexpr int kHistPadded = 32 * (kHistBins / 32 + 1);

__device__ __forceinline__ ThresholdPick pick_threshold_shared(const Problem& pb, double mag, const double* s_s2,
                                                               const unsigned long long* s_cnt)
{
    constexpr int kPer = kHistBins / 32;
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const double k = pb.comps == 1 ? 2.0 * pb.n : 6.0 * pb.n;
    const double var_per_s2 = mul_rn(k / 12.0, 0x1p-104);
    const double half = mul_rn(0.5 * pb.tol, mag);
    const double budget = mag > 0.0 ? mul_rn(half, half) : 0.0;
    double v[kPer];
    unsigned long long cn[kPer];
    double loc = 0.0;
    unsigned long long cl = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int b = lane * kPer + i;
        v[i] = mul_rn(s_s2[hist_pad_index(b)], var_per_s2);
        cn[i] = s_cnt[hist_pad_index(b)];
        loc = add_rn(loc, v[i]);
        cl += cn[i];
    }
    // Inclusive prefix of the lanes' sums of v, inclusive suffix of their counts.
    double incl = loc;
    unsigned long long sfx = cl;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double o = __shfl_up_sync(full, incl, d);
        const unsigned long long p = __shfl_down_sync(full, sfx, d);
        if (lane >= d) incl = add_rn(incl, o);
        if (lane + d < 32) sfx += p;
    }
    double excl = __shfl_up_sync(full, incl, 1);
    if (lane == 0) excl = 0.0;
    unsigned long long after = __shfl_down_sync(full, sfx, 1);  // units in the lanes above
    if (lane == 31) after = 0;
    // b0: the first bin whose cumulative sum would exceed the budget.
    int first = kHistBins;
    double cum = excl;
#pragma unroll
    for (int i = 0; i < kPer; ++i)
        if (first == kHistBins) {
            const double next = add_rn(cum, v[i]);
            if (!(next <= budget)) first = lane * kPer + i;
            else cum = next;
        }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) first = min(first, __shfl_xor_sync(full, first, d));
    // b: the first bin >= b0 whose tail holds at most units/8 units.
    const unsigned long long cap = pb.units / 8;
    int bsel = kHistBins;
    unsigned long long tail = after;  // units in bins >= the current one, walking down
#pragma unroll
    for (int i = kPer - 1; i >= 0; --i) {
        tail += cn[i];
        const int bin = lane * kPer + i;
        if (bin >= first && tail <= cap) bsel = bin;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) bsel = min(bsel, __shfl_xor_sync(full, bsel, d));
    // The owner of bin bsel (lane 31 for bsel == kHistBins) has the sums below it.
    const int owner = bsel < kHistBins ? bsel / kPer : 31;
    double below = excl;
    unsigned long long from = after;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int bin = lane * kPer + i;
        if (bin < bsel) below = add_rn(below, v[i]);
        else from += cn[i];
    }
    below = __shfl_sync(full, below, owner);
    from = __shfl_sync(full, from, owner);
    ThresholdPick t;
    t.thr = bsel;
    t.count = bsel < kHistBins ? from : 0ull;
    t.err = mag > 0.0 ? sqrt(below) / mag : INFINITY;
    return t;
}

}  // namespace dense
}  // namespace spb
