// Double-double re-evaluation of the dominant units (precision SPB_PREC_DD).
//
// Ryser's alternating sum is dominated, for many inputs, by a small set of
// very large terms (for positive matrices: subsets near the empty and the
// full set).  Their FP64 rounding errors, not the many small terms, set the
// final error.  The walk (mode 1) bins every unit by an upper bound U_u of its
// terms and accumulates the unit's actual sum of squared terms in that bin;
// dd_threshold picks the bin from which the remaining units' rounding error
// fits the tolerance.  The units at or above it come from the walk's own list
// (every unit at or above a bin chosen beforehand by bound_walk, when that
// bin is low enough), else from a parallel scan (list_units does either), and
// only if either count disagrees with the histogram from a replay scan (walk mode 2,
// same launch shape, so the unit bases are bit-identical) that lists them
// with their double-double base vectors.  This kernel then re-evaluates each
// listed unit on a worker of one or more warps:
//   * the FP64 unit sum exactly as the walk computed it (same operations in
//     the same order, so the same bits), spread over the lanes by group;
//   * the double-double unit sum (x_r = xtop_r + DE[d][r] in double-double,
//     double-double products and sum);
// and accumulates sign_u * (dd_sum - fp64_sum) into pb.result.  Adding that
// correction to the walk's total replaces the dominant units' FP64 values by
// their double-double values.
#include <mutex>

#include "bound_impl.cuh"
#include "dense_impl.cuh"
#include "refine_impl.cuh"

namespace spb {
namespace dense {
namespace {

// One group of G (<= 4) complex terms, bitwise identical to unit_sum_complex<N,G>.
// The group's term i of row r is dr/di[r * rs + i].
__device__ __forceinline__ void group_sum_complex_rt(const double* xr, const double* xi,
                                                     const double* dr, const double* di, int n,
                                                     int G, int rs, double& gr, double& gi)
{
    double pr[4] = {0.0, 0.0, 0.0, 0.0}, pi[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < G; ++i) {
        pr[i] = add_rn(xr[0], dr[i]);
        pi[i] = add_rn(xi[0], di[i]);
    }
    for (int r = 1; r < n; ++r) {
        for (int i = 0; i < G; ++i) {
            double yr = add_rn(xr[r], dr[r * rs + i]);
            double yi = add_rn(xi[r], di[r * rs + i]);
            double t1 = mul_rn(pi[i], yi);
            double t2 = mul_rn(pi[i], yr);
            double nr = __fma_rn(pr[i], yr, -t1);
            double ni = __fma_rn(pr[i], yi, t2);
            pr[i] = nr;
            pi[i] = ni;
        }
    }
    if (G == 4) {
        gr = sub_rn(sub_rn(pr[0], pr[1]), sub_rn(pr[2], pr[3]));
        gi = sub_rn(sub_rn(pi[0], pi[1]), sub_rn(pi[2], pi[3]));
    } else if (G == 2) {
        gr = sub_rn(pr[0], pr[1]);
        gi = sub_rn(pi[0], pi[1]);
    } else {
        gr = pr[0];
        gi = pi[0];
    }
}

// Unit base of unit u (component `part`) rebuilt from scratch in
// double-double the way the walk builds a thread's first unit (x0 plus the
// selected high columns in index order); the worker's threads take rows.
__device__ __forceinline__ void unit_base(const Problem& pb, const double* mt_all, unsigned long long u, int part,
                                          int lane, double* hi, double* lo, int stride = 32)
{
    const int n = pb.n, ntop = n - 1 - pb.w;
    const unsigned long long g = gray_of(u);
    const double* mt = mt_all + (size_t)part * (ntop > 0 ? ntop : 0) * n;
    for (int r = lane; r < n; r += stride) {
        dd x = {pb.x0_hi[part * n + r], pb.x0_lo[part * n + r]};
        for (int j = 0; j < ntop; ++j)
            if ((g >> j) & 1ull) x = dd_add_d(x, mt[j * n + r]);
        hi[r] = x.hi;
        lo[r] = x.lo;
    }
}

// The walk's unit bound (dense_impl.cuh walk_real/walk_complex, and
// sparse_impl.cuh walk_sparse when pb.na < pb.n) from the hi words of a unit
// base (xh: [comps][n]): the same operations in the same order.
__device__ double unit_bound_rt(const Problem& pb, const double* xh)
{
    const int n = pb.n, na = pb.na;
    double ub = 1.0;
    if (pb.comps == 2) {
        for (int r = 0; r < n; ++r) {
            const double xr = xh[r], xi = xh[kMaxN + r];
            ub = mul_rn(ub, add_rn(__dsqrt_rn(__fma_rn(xr, xr, mul_rn(xi, xi))), pb.bnd[r]));
        }
        return ub;
    }
    if (na < n) {
        double c = xh[na];
        for (int r = na + 1; r < n; ++r) c = mul_rn(c, xh[r]);
        ub = fabs(c);
    }
    for (int r = 0; r < na; ++r)
        ub = mul_rn(ub, fmax(fabs(add_rn(xh[r], pb.bnd[r])), fabs(add_rn(xh[r], pb.bnd[n + r]))));
    return ub;
}

// Lists the units whose bin >= rb->thr, unit indices only (the refine kernel
// rebuilds the bases).  When the walk's own list holds all of them
// (rb->from_list), every thread keeps the listed units at or above rb->thr.
// Otherwise the walk's threads whose highest bin reaches it (tmax) are
// visited one per warp; each lane
// takes a contiguous part of that thread's units, builds the first unit base
// from scratch in double-double and steps through the Gray order with the
// walk's own base update, evaluating the walk's bound per unit.  A lane's bases start
// from a rebuild rather than from the walk's thread start, so a hi word could
// in principle differ from the walk's (a row value within ~2^-100 of a
// rounding midpoint); if that ever moved a unit across the threshold the
// count check fails and the caller falls back to the replay scan.
__global__ void __launch_bounds__(128) list_units(Problem pb)
{
    if (pb.rb->count == 0) return;
    const int thr = pb.rb->thr;
    if (pb.rb->from_list) {
        const unsigned long long m = *pb.raw_n < pb.raw_cap ? *pb.raw_n : pb.raw_cap;
        for (unsigned long long e = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; e < m;
             e += (unsigned long long)gridDim.x * blockDim.x)
            if ((int)pb.raw_b[e] >= thr) {
                const unsigned long long i = atomicAdd(pb.list_n, 1ull);
                if (i < pb.list_cap) pb.list_u[i] = pb.raw_u[e];
            }
        return;
    }
    const unsigned long long T = (unsigned long long)pb.grid * pb.threads;
    const int lane = threadIdx.x & 31, n = pb.n, c = pb.comps;
    const int ntop = n - 1 - pb.w, ntp = ntop > 0 ? ntop : 0;
    const unsigned long long warp = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned long long nwarps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    double xh[2 * kMaxN], xl[2 * kMaxN];  // [comps][kMaxN], per lane
    for (unsigned long long t = warp; t < T; t += nwarps) {
        if ((int)pb.tmax[t] < thr) continue;  // warp-uniform
        unsigned long long u0, u1;
        balanced_range(pb.units, T, t, &u0, &u1);
        unsigned long long a, b;
        balanced_range(u1 - u0, 32, lane, &a, &b);
        a += u0;
        b += u0;
        if (a >= b) continue;
        const unsigned long long g0 = gray_of(a);
        for (int part = 0; part < c; ++part) {
            const double* mt = pb.mt + (size_t)part * ntp * n;
            for (int r = 0; r < n; ++r) {
                dd x = {pb.x0_hi[part * n + r], pb.x0_lo[part * n + r]};
                for (int j = 0; j < ntop; ++j)
                    if ((g0 >> j) & 1ull) x = dd_add_d(x, mt[j * n + r]);
                xh[part * kMaxN + r] = x.hi;
                xl[part * kMaxN + r] = x.lo;
            }
        }
        for (unsigned long long u = a;;) {
            if (hist_bin(unit_bound_rt(pb, xh)) >= thr) {
                const unsigned long long i = atomicAdd(pb.list_n, 1ull);
                if (i < pb.list_cap) pb.list_u[i] = u;
            }
            if (++u >= b) break;
            const int j = __ffsll((long long)u) - 1;
            const bool add = (gray_of(u) >> j) & 1ull;
            for (int part = 0; part < c; ++part) {
                const double* col = pb.mt + ((size_t)part * ntp + j) * n;
                for (int r = 0; r < n; ++r) {
                    const double m = add ? col[r] : -col[r];
                    dd s = two_sum(xh[part * kMaxN + r], m);
                    dd z = fast_two_sum(s.hi, add_rn(s.lo, xl[part * kMaxN + r]));
                    xh[part * kMaxN + r] = z.hi;
                    xl[part * kMaxN + r] = z.lo;
                }
            }
        }
    }
}

// *list_bin = the lowest bin whose tail (units at or above it) holds
// at most kRawTarget units by bound_walk's count.  One warp; lane l owns bins
// [16l, 16l + 16) and the tails are lane-local sums joined by a warp scan.
// The counts are staged in shared memory with coalesced loads first.
__global__ void __launch_bounds__(32) pick_list_bin(Problem pb)
{
    constexpr int kPer = kHistBins / 32;
    const int lane = threadIdx.x;
    const unsigned full = 0xffffffffu;
    __shared__ unsigned s_pc[kHistPadded];
    {
        // all of a lane's loads issued before the first store (one L2
        // latency, not kPer of them in a row)
        unsigned v[kPer];
#pragma unroll
        for (int i = 0; i < kPer; ++i) v[i] = __ldcg(pb.pre_cnt + lane + 32 * i);
#pragma unroll
        for (int i = 0; i < kPer; ++i) s_pc[hist_pad_index(lane + 32 * i)] = v[i];
    }
    __syncwarp();
    unsigned long long cn[kPer], cl = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        cn[i] = s_pc[hist_pad_index(lane * kPer + i)];
        cl += cn[i];
    }
    unsigned long long sfx = cl;  // inclusive suffix over lanes
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long p = __shfl_down_sync(full, sfx, d);
        if (lane + d < 32) sfx += p;
    }
    unsigned long long tail = __shfl_down_sync(full, sfx, 1);
    if (lane == 31) tail = 0;
    const unsigned long long target = kRawTarget;
    int b = kHistBins;
#pragma unroll
    for (int i = kPer - 1; i >= 0; --i) {
        tail += cn[i];
        if (tail <= target) b = lane * kPer + i;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) b = min(b, __shfl_xor_sync(full, b, d));
    if (lane == 0) *pb.list_bin = b;
}

// Picks the refinement bin (pick_threshold, refine_impl.cuh) from the walk's
// histogram and total.  Also decides whether the walk's own list holds every
// unit at or above it (no overflow, bin >= its list bin) and resets the list
// counter.  One warp.
__global__ void __launch_bounds__(32) dd_threshold(Problem pb)
{
    const int lane = threadIdx.x;
    Readback* rb = pb.rb;
    // the histogram staged in shared memory with coalesced loads (read in
    // place, each lane's 16 consecutive bins cost one L2 request per bin)
    __shared__ double s_h2[kHistPadded];
    __shared__ unsigned long long s_hc[kHistPadded];
    {
        // all of a lane's loads issued before the first store (one L2
        // latency, not 16 of them in a row)
        constexpr int kPer = kHistBins / 32;
        double v2[kPer];
        unsigned long long vc[kPer];
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            v2[i] = __ldcg(pb.hist_s2 + lane + 32 * i);
            vc[i] = __ldcg(pb.hist_cnt + lane + 32 * i);
        }
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            s_h2[hist_pad_index(lane + 32 * i)] = v2[i];
            s_hc[hist_pad_index(lane + 32 * i)] = vc[i];
        }
    }
    __syncwarp();
    const double mag = pb.comps == 1 ? fabs(rb->res[0].hi) : hypot(rb->res[0].hi, rb->res[1].hi);
    const ThresholdPick t = pick_threshold_shared(pb, mag, s_h2, s_hc);
    if (lane == 0) {
        rb->thr = t.thr;
        rb->count = t.count;
        rb->err = t.err;
        rb->from_list = (t.thr >= *pb.list_bin && *pb.raw_n <= pb.raw_cap) ? 1 : 0;
        rb->list_n = 0;
        // the refinement writes its correction only when it has units
        rb->corr[0] = dd{0.0, 0.0};
        rb->corr[1] = dd{0.0, 0.0};
    }
}

// Units to refine: the histogram's count when the listing found exactly
// that many and the list held them all, else none (the host then lists
// again and reruns the refinement).  With none, the refine kernels return at
// once (the count is the same for every CTA) and rb->corr keeps the zero
// dd_threshold wrote.
__device__ __forceinline__ unsigned long long refine_count(const Problem& pb)
{
    const unsigned long long want = pb.rb->count;
    return (pb.rb->list_n == want && want <= pb.list_cap) ? want : 0ull;
}

// Copies m doubles from global to shared memory, eight loads in flight per
// thread (a plain loop waits out one global-memory latency per element).
__device__ __forceinline__ void stage(double* dst, const double* __restrict__ src, int m)
{
    const int bd = blockDim.x;
    for (int i0 = threadIdx.x; i0 < m; i0 += 8 * bd) {
        double v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int i = i0 + k * bd;
            v[k] = i < m ? __ldg(src + i) : 0.0;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int i = i0 + k * bd;
            if (i < m) dst[i] = v[k];
        }
    }
}

// Copies `parts` subset-sum tables laid out [q][n][G] (the walks' grouping,
// q = d / G) into shared memory as [n][terms] (d contiguous per row), so
// that lanes taking consecutive terms of one row read consecutive words
// rather than words n*G apart in one bank.  For even G the threads move
// 16-byte pairs in destination order: consecutive lanes write consecutive
// pairs of one row (no bank conflicts; the transposed order put a warp's
// stores 8*terms bytes apart, all in one bank) and read half of one 32-byte
// group each, eight pairs in flight per thread.
__device__ __forceinline__ void stage_rows(double* dst, const double* __restrict__ src, int parts, int n,
                                           int terms, int G)
{
    const int per = terms * n, bd = blockDim.x;
    if (G == 1) {  // n < 3: tiny tables
        for (int i = threadIdx.x; i < parts * per; i += bd) {
            const int part = i / per, rd = i % per, r = rd / terms, d = rd % terms;
            dst[i] = src[(size_t)part * per + (size_t)d * n + r];
        }
        return;
    }
    // terms is a power of two and G is 2 or 4, so the index splits by shifts
    // and masks; parts is 1 or 2 (no division by n either)
    const int half = terms / 2, total = parts * n * half;  // pairs per row, all
    const int lh = __ffs(half) - 1, lp = G == 4 ? 1 : 0;    // log2 half, log2 pairs per group
    const double2* s2 = reinterpret_cast<const double2*>(src);
    double2* d2 = reinterpret_cast<double2*>(dst);
    for (int t0 = threadIdx.x; t0 < total; t0 += 8 * bd) {
        double2 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int t = t0 + k * bd;
            if (t < total) {
                // t = (part * n + r) * half + c, c = q * (G / 2) + h
                const int pr = t >> lh, c = t & (half - 1), part = pr >= n ? 1 : 0, r = pr - part * n;
                const int q = c >> lp, h = c & lp;
                v[k] = __ldg(s2 + ((size_t)part * per + ((size_t)q * n + r) * G) / 2 + h);
            }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int t = t0 + k * bd;
            if (t < total) d2[t] = v[k];
        }
    }
}

// Threads per refinement worker: a warp, doubled while every unit still
// gets its own worker in one round over the grid's warps and each thread
// keeps at least `per_lane` terms (two independent chains in the real
// kernel, one in the complex).  Few units then spread over many warps
// instead of leaving most of the grid idle behind a few long chains.
__device__ __forceinline__ int refine_worker_threads(unsigned long long count, int terms, int per_lane)
{
    const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x >> 5);
    int wk = 32;
    while (2 * wk <= (int)blockDim.x && 2 * wk * per_lane <= terms && count * (unsigned long long)(2 * wk / 32) <= warps)
        wk *= 2;
    return wk;
}

// Sums a dd over a worker of wk threads (warp sums added in warp order
// through s_red).  The result is valid in the worker's thread 0.  Every
// thread of the CTA calls it when wk > 32 (it holds a block barrier).
__device__ __forceinline__ dd worker_sum_dd(dd v, int wk, dd* s_red)
{
    v = warp_sum_dd(v);
    if (wk == 32) return v;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s_red[wid] = v;
    __syncthreads();
    if (threadIdx.x % wk == 0)
        for (int i = 1; i < wk / 32; ++i) v = dd_add(v, s_red[wid + i]);
    return v;
}

__device__ __forceinline__ void worker_sync(int wk)
{
    if (wk > 32) __syncthreads();
    else __syncwarp();
}

// A unit is refined by a worker of wk threads (refine_worker_threads).
// Units are dealt out CTA by CTA (unit e to CTA e mod grid), so that a few
// hundred units occupy every SM rather than filling a few.  The loop runs in
// rounds of one unit per worker, the same number of rounds in every CTA, so
// that the block barriers of multi-warp workers are met by all threads.  A
// worker's threads take terms; each runs two independent term chains at a
// time when it has two.
__global__ void __launch_bounds__(512, 1) refine_real(Problem pb)
{
    const unsigned long long count = refine_count(pb);
    if (count == 0) return;
    extern __shared__ __align__(16) double sm[];
    __shared__ dd s_red[16];
    const int n = pb.n, G = pb.g, terms = 1 << pb.w, nq = terms / G;
    const int nwarps = blockDim.x >> 5;
    const int wk = refine_worker_threads(count, terms, 2);  // threads per worker
    const int wl = threadIdx.x % wk, wid = threadIdx.x / wk, nwk = blockDim.x / wk;
    const int ntp = n - 1 - pb.w > 0 ? n - 1 - pb.w : 0;
    double* s_dh = sm;
    double* s_dl = s_dh + terms * n;
    double* s_x = s_dl + terms * n;      // [nwarps][2n]
    double* s_g = s_x + nwarps * 2 * n;  // [nwarps][nq]
    double* s_mt = s_g + nwarps * nq;    // [ntp][n]
    // CTAs without a unit skip the tables (they still join the grid reduction)
    if ((unsigned long long)blockIdx.x < count) {
        stage_rows(s_dh, pb.de_hi, 1, n, terms, G);  // [n][terms]
        stage_rows(s_dl, pb.de_lo, 1, n, terms, G);
        stage(s_mt, pb.mt, ntp * n);
    }
    __syncthreads();
    double* xw = s_x + wid * 2 * n;
    double* gw = s_g + wid * nq;
    dd corr = {0.0, 0.0};
    const unsigned long long round = (unsigned long long)gridDim.x * nwk;
    for (unsigned long long e0 = 0; e0 < count; e0 += round) {
        const unsigned long long e = e0 + (unsigned long long)wid * gridDim.x + blockIdx.x;
        const bool active = e < count;
        if (active) {
            if (pb.list_x) {
                const double* src = pb.list_x + e * (2 * n);
                for (int i = wl; i < 2 * n; i += wk) xw[i] = src[i];
            } else {
                unit_base(pb, s_mt, pb.list_u[e], 0, wl, xw, xw + n, wk);
            }
        }
        worker_sync(wk);
        dd acc = {0.0, 0.0};
        if (active) {
            for (int q = wl; q < nq; q += wk) gw[q] = group_sum_real_rt(xw, s_dh + q * G, n, pb.na, G, terms);
            if (terms >= 2 * wk) {
                for (int d = wl; d < terms; d += 2 * wk) {
                    const int d2 = d + wk;
                    dd p1 = dd_add_fast(dd{xw[0], xw[n]}, dd{s_dh[d], s_dl[d]});
                    dd p2 = dd_add_fast(dd{xw[0], xw[n]}, dd{s_dh[d2], s_dl[d2]});
                    int r = 1;
                    // four rows' factors formed ahead of the products (they
                    // do not depend on them), then multiplied in row order
                    for (; r + 3 < n; r += 4) {
                        dd y1[4], y2[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const int k1 = (r + k) * terms + d, k2 = (r + k) * terms + d2;
                            const dd x = {xw[r + k], xw[n + r + k]};
                            y1[k] = dd_add_fast(x, dd{s_dh[k1], s_dl[k1]});
                            y2[k] = dd_add_fast(x, dd{s_dh[k2], s_dl[k2]});
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            p1 = dd_mul(p1, y1[k]);
                            p2 = dd_mul(p2, y2[k]);
                        }
                    }
                    for (; r < n; ++r) {
                        const int k1 = r * terms + d, k2 = r * terms + d2;
                        const dd x = {xw[r], xw[n + r]};
                        p1 = dd_mul(p1, dd_add_fast(x, dd{s_dh[k1], s_dl[k1]}));
                        p2 = dd_mul(p2, dd_add_fast(x, dd{s_dh[k2], s_dl[k2]}));
                    }
                    acc = (__popc(d) & 1) ? dd_add(acc, dd_neg(p1)) : dd_add(acc, p1);
                    acc = (__popc(d2) & 1) ? dd_add(acc, dd_neg(p2)) : dd_add(acc, p2);
                }
            } else {
                for (int d = wl; d < terms; d += wk) {
                    dd p = dd_add_fast(dd{xw[0], xw[n]}, dd{s_dh[d], s_dl[d]});
                    int r = 1;
                    for (; r + 3 < n; r += 4) {
                        dd y[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const int i = (r + k) * terms + d;
                            y[k] = dd_add_fast(dd{xw[r + k], xw[n + r + k]}, dd{s_dh[i], s_dl[i]});
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k) p = dd_mul(p, y[k]);
                    }
                    for (; r < n; ++r) {
                        const int k = r * terms + d;
                        p = dd_mul(p, dd_add_fast(dd{xw[r], xw[n + r]}, dd{s_dh[k], s_dl[k]}));
                    }
                    acc = (__popc(d) & 1) ? dd_add(acc, dd_neg(p)) : dd_add(acc, p);
                }
            }
        }
        acc = worker_sum_dd(acc, wk, s_red);
        worker_sync(wk);
        if (active && wl == 0) {
            double f = 0.0;
            for (int q = 0; q < nq; ++q) f = (__popc(q) & 1) ? sub_rn(f, gw[q]) : add_rn(f, gw[q]);
            dd c = dd_add_d(acc, -f);
            if (pb.list_u[e] & 1ull) c = dd_neg(c);
            corr = dd_add(corr, c);
        }
        worker_sync(wk);
    }
    dd tot[1] = {corr};
    grid_reduce<1>(tot, pb);
}

__global__ void __launch_bounds__(512, 1) refine_complex(Problem pb)
{
    const unsigned long long count = refine_count(pb);
    if (count == 0) return;
    extern __shared__ __align__(16) double sm[];
    __shared__ dd s_red[2][16];
    const int n = pb.n, G = pb.g, terms = 1 << pb.w, nq = terms / G;
    const int nwarps = blockDim.x >> 5;
    const int wk = refine_worker_threads(count, terms, 1);  // threads per worker
    const int wl = threadIdx.x % wk, wid = threadIdx.x / wk, nwk = blockDim.x / wk;
    const int ntp = n - 1 - pb.w > 0 ? n - 1 - pb.w : 0;
    double* s_dh = sm;                    // [2][terms*n]
    double* s_dl = s_dh + 2 * terms * n;  // [2][terms*n]
    double* s_x = s_dl + 2 * terms * n;   // [nwarps][4n]
    double* s_g = s_x + nwarps * 4 * n;   // [nwarps][2*nq]
    double* s_mt = s_g + nwarps * 2 * nq; // [2][ntp][n]
    // CTAs without a unit skip the tables (they still join the grid reduction)
    if ((unsigned long long)blockIdx.x < count) {
        stage_rows(s_dh, pb.de_hi, 2, n, terms, G);  // [2][n][terms]
        stage_rows(s_dl, pb.de_lo, 2, n, terms, G);
        stage(s_mt, pb.mt, 2 * ntp * n);
    }
    __syncthreads();
    const double* drh = s_dh;
    const double* dih = s_dh + terms * n;
    const double* drl = s_dl;
    const double* dil = s_dl + terms * n;
    double* xw = s_x + wid * 4 * n;  // xr hi, xr lo, xi hi, xi lo
    double* gw = s_g + wid * 2 * nq;
    dd corr_r = {0.0, 0.0}, corr_i = {0.0, 0.0};
    const unsigned long long round = (unsigned long long)gridDim.x * nwk;
    for (unsigned long long e0 = 0; e0 < count; e0 += round) {
        const unsigned long long e = e0 + (unsigned long long)wid * gridDim.x + blockIdx.x;
        const bool active = e < count;
        if (active) {
            if (pb.list_x) {
                const double* src = pb.list_x + e * (4 * n);
                for (int i = wl; i < 4 * n; i += wk) xw[i] = src[i];
            } else {
                unit_base(pb, s_mt, pb.list_u[e], 0, wl, xw, xw + n, wk);
                unit_base(pb, s_mt, pb.list_u[e], 1, wl, xw + 2 * n, xw + 3 * n, wk);
            }
        }
        worker_sync(wk);
        dd ar = {0.0, 0.0}, ai = {0.0, 0.0};
        if (active) {
            for (int q = wl; q < nq; q += wk)
                group_sum_complex_rt(xw, xw + 2 * n, drh + q * G, dih + q * G, n, G, terms, gw[2 * q],
                                     gw[2 * q + 1]);
            for (int d = wl; d < terms; d += wk) {
                int k = d;
                dd pr = dd_add_fast(dd{xw[0], xw[n]}, dd{drh[k], drl[k]});
                dd pi = dd_add_fast(dd{xw[2 * n], xw[3 * n]}, dd{dih[k], dil[k]});
                for (int r = 1; r < n; ++r) {
                    k = r * terms + d;
                    dd yr = dd_add_fast(dd{xw[r], xw[n + r]}, dd{drh[k], drl[k]});
                    dd yi = dd_add_fast(dd{xw[2 * n + r], xw[3 * n + r]}, dd{dih[k], dil[k]});
                    // the products' sums unnormalised (dd_add_fast: about 2^-106 of
                    // |pr yr| + |pi yi| off, far inside what the refinement corrects)
                    dd nr = dd_add_fast(dd_mul(pr, yr), dd_neg(dd_mul(pi, yi)));
                    dd ni = dd_add_fast(dd_mul(pr, yi), dd_mul(pi, yr));
                    pr = nr;
                    pi = ni;
                }
                if (__popc(d) & 1) {
                    ar = dd_add(ar, dd_neg(pr));
                    ai = dd_add(ai, dd_neg(pi));
                } else {
                    ar = dd_add(ar, pr);
                    ai = dd_add(ai, pi);
                }
            }
        }
        ar = worker_sum_dd(ar, wk, s_red[0]);
        ai = worker_sum_dd(ai, wk, s_red[1]);
        worker_sync(wk);
        if (active && wl == 0) {
            double fr = 0.0, fi = 0.0;
            for (int q = 0; q < nq; ++q) {
                if (__popc(q) & 1) {
                    fr = sub_rn(fr, gw[2 * q]);
                    fi = sub_rn(fi, gw[2 * q + 1]);
                } else {
                    fr = add_rn(fr, gw[2 * q]);
                    fi = add_rn(fi, gw[2 * q + 1]);
                }
            }
            dd cr = dd_add_d(ar, -fr), ci = dd_add_d(ai, -fi);
            if (pb.list_u[e] & 1ull) {
                cr = dd_neg(cr);
                ci = dd_neg(ci);
            }
            corr_r = dd_add(corr_r, cr);
            corr_i = dd_add(corr_i, ci);
        }
        worker_sync(wk);
    }
    dd tot[2] = {corr_r, corr_i};
    grid_reduce<2>(tot, pb);
}

}  // namespace

template <int N>
int launch_bound_n(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s);

int launch_bound_pass(const Problem& pb, int blocks, cudaStream_t s)
{
    const int threads = 256;
    const size_t smem = bound_smem_bytes_f(pb.n, pb.comps, pb.w);
    // Two CTAs per SM, but at least 8 units per thread: a thread's first
    // unit base costs n*(n-1-w) adds, so few units per thread would be
    // dominated by that start.
    blocks *= 2;
    unsigned long long max_blocks = (pb.units + 8ull * threads - 1) / (8ull * threads);
    if ((unsigned long long)blocks > max_blocks) blocks = (int)max_blocks;
    if (blocks < 1) blocks = 1;
    int st = SPB_ERR_INVALID;
    switch (pb.n) {
#define SPB_CASE(N) \
    case N: st = launch_bound_n<N>(pb, blocks, threads, smem, s); break;
        SPB_FOR_EACH_N(SPB_CASE)
#undef SPB_CASE
    default:
        spb_set_error("bound pass: n=%d outside 1..%d", pb.n, kMaxN);
        return SPB_ERR_INVALID;
    }
    if (st != SPB_OK) return st;
    pick_list_bin<<<1, 32, 0, s>>>(pb);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

int launch_listing(const Problem& pb, cudaStream_t s)
{
    list_units<<<pb.grid * 4, 128, 0, s>>>(pb);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

int launch_threshold(const Problem& pb, cudaStream_t s)
{
    dd_threshold<<<1, 32, 0, s>>>(pb);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

size_t refine_smem_bytes(const Problem& pb, int threads)
{
    const size_t terms = (size_t)1 << pb.w, n = pb.n, c = pb.comps, nq = terms / pb.g;
    const size_t nwarps = threads / 32;
    const size_t ntp = pb.n - 1 - pb.w > 0 ? pb.n - 1 - pb.w : 0;
    return sizeof(double) * (2 * c * terms * n + nwarps * (2 * c * n + c * nq) + c * ntp * n);
}

int launch_refine(const Problem& pb, int blocks, cudaStream_t s)
{
    // 512 threads (16 warps per SM hide the double-double latency chains)
    // when their per-warp buffers fit next to the tables, else 256.
    int threads = 512;
    size_t smem = refine_smem_bytes(pb, threads);
    const int ck = pb.comps == 1 ? 0 : 1;
    auto kern = ck == 0 ? refine_real : refine_complex;
    // The shared-memory limit is raised once per device and kernel.
    static std::mutex mu;
    static int limit[64][2];
    int dev = 0;
    SPB_CUDA_TRY(cudaGetDevice(&dev));
    int room = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev < 0 || dev >= 64) {
            spb_set_error("refine: device %d out of range", dev);
            return SPB_ERR_INVALID;
        }
        if (limit[dev][ck] == 0) {
            int optin = 0;
            cudaFuncAttributes fa{};
            SPB_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
            SPB_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
            SPB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              optin - (int)fa.sharedSizeBytes));
            limit[dev][ck] = optin - (int)fa.sharedSizeBytes;
        }
        room = limit[dev][ck];
    }
    if (smem > (size_t)room) {
        threads = 256;
        smem = refine_smem_bytes(pb, threads);
    }
    if (smem > (size_t)room) {
        spb_set_error("refine: n=%d needs %zu B shared memory", pb.n, smem);
        return SPB_ERR_INVALID;
    }
    Problem pr = pb;
    pr.result = pb.rb->corr;
    kern<<<blocks, threads, smem, s>>>(pr);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

}  // namespace dense
}  // namespace spb
