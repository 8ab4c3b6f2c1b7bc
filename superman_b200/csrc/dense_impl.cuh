// Dense walk kernels (real and complex), shared between the driver in
// dense.cu and the per-n instantiation units dense_walk_{real,complex}.cu.
#pragma once

#include <cuda_runtime.h>

#include "spb_common.cuh"

namespace spb {
namespace dense {

constexpr int kMaxN = 63;

// Everything the host reads back after a call, contiguous so that one copy
// brings it over: a call costs one host round trip, the double-double
// refinement included (its threshold is picked on the device).
struct Readback {
    dd res[2];                  // [comps] the walk's total
    dd corr[2];                 // [comps] the refinement's correction
    unsigned long long list_n;  // units listed for the refinement
    unsigned long long count;   // units the histogram puts at or above thr
    double err;                 // SPB_PREC_DD: expected relative error of the unrefined units;
                                // SPB_PREC_FP32: the walk's sum of squared terms
    int thr;                    // refinement bin
    int from_list;              // 1: the walk's own list holds every unit at or above thr
    int exp_sum;                // sum of the row scaling exponents
    int pad;
};

// Device-side description of one permanent: sizes plus pointers into the
// scratch arena written by setup_kernel.
struct Problem {
    int n, comps, w, g, grid, threads;
    int na;                    // rows that vary within a unit: n (dense walk) or the
                               // active rows of the row-compacted walk (sparse_impl.cuh)
    unsigned long long units;  // 2^(n-1-w) Gray units of 2^w terms each
    double* as;                // row-scaled matrix (row-major, comps interleaved)
    double* x0_hi;             // [comps][n] NW start vector, double-double
    double* x0_lo;
    double* de_hi;             // [comps][2^w/G][n][G] low-column subset sums
    double* de_lo;             // rounding residues of de_hi
    float* de32;               // SPB_PREC_FP32: de_hi rounded to float (else null)
    int f32;                   // 1: the FP32-product walk runs (tables include de32)
    double* mt;                // [comps][n-1-w][n] high columns
    dd* partials;              // [comps][grid] per-CTA sums
    unsigned* ticket;          // last-CTA election counter (reset by the kernel)
    dd* result;                // [comps] grid total (rb->res; rb->corr for the refinement)
    int* exp_sum;              // sum of the row scaling exponents (&rb->exp_sum)
    Readback* rb;
    double tol;                // SPB_PREC_DD: relative tolerance of the threshold
    // Double-double refinement (SPB_PREC_DD); unused when mode == 0.
    int mode;                  // 0 walk, 1 walk + unit-bound histogram, 2 scan only
    int thr_bin;               // mode 2: list the units whose bound bin >= thr_bin
    double* bnd;               // real [2][n] min/max of DE over d; complex [n] max |DE|
    double* hist_s2;           // [kHistBins] sum of squared terms of the units per bin
    unsigned long long* hist_cnt;  // [kHistBins] units per bin
    unsigned long long* list_n;    // number of listed units (&rb->list_n)
    unsigned long long list_cap;
    unsigned long long* list_u;    // [list_cap] unit index
    double* list_x;                // [list_cap][comps][2][n] unit base, hi then lo
    unsigned short* tmax;          // [grid*threads] highest bound bin of each thread's units
    // Mode 1 direct listing: bound_walk counts the units per bound bin
    // (pre_cnt), pick_list_bin sets *list_bin to the lowest bin whose tail fits
    // raw_cap, and the walk appends every unit at or above it (raw_*).
    unsigned* pre_cnt;             // [kHistBins]
    int* list_bin;
    int list_bin_init;             // written to *list_bin by setup_kernel (pick_list_bin may overwrite it)
    unsigned long long* raw_n;
    unsigned long long raw_cap;
    unsigned long long* raw_u;     // [raw_cap] unit index
    unsigned short* raw_b;         // [raw_cap] its bound bin
};

// Capacity of the mode-1 list (units; 10 bytes each, 21 MB).  A walk of at
// most kRawCap / 2 units (real n <= 29, complex n <= 28 at the default unit
// width) lists every unit and needs no bound pass; larger walks list from
// the bin pick_list_bin chooses, aiming at kRawTarget units, far below the
// capacity so that bins computed by the walk and by bound_walk may differ at
// bin edges.  The units the refinement takes (a few hundred to a few thousand
// from n = 27 to 32) fit that target many times over, and every listed unit
// costs the walk an append.
constexpr unsigned long long kRawCap = 1ull << 21;
constexpr unsigned long long kRawTarget = 1ull << 14;

// Appends unit u (bound bin b) to the mode-1 list when b >= lbin.  The
// appending lanes of a warp take their slots with one atomic (a leader
// reserves popc of them), not one each.
__device__ __forceinline__ void raw_list_add(const Problem& pb, int lbin, unsigned long long u, int b)
{
    const unsigned act = __activemask();
    const bool want = b >= lbin;
    const unsigned m = __ballot_sync(act, want);
    if (!want) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(pb.raw_n, (unsigned long long)__popc(m));
    base = __shfl_sync(m, base, leader);
    const unsigned long long k = base + (unsigned long long)__popc(m & ((1u << lane) - 1u));
    if (k < pb.raw_cap) {
        pb.raw_u[k] = u;
        pb.raw_b[k] = (unsigned short)b;
    }
}

// Unit-bound histogram: bin = (ilogb(U) + 1024) / 4, i.e. four octaves per bin.
constexpr int kHistBins = 512;

__device__ __forceinline__ int hist_bin(double u)
{
    if (!(u > 0.0)) return 0;
    if (!isfinite(u)) return kHistBins - 1;
    int b = (ilogb(u) + 1024) >> 2;
    return b < 0 ? 0 : (b >= kHistBins ? kHistBins - 1 : b);
}

// Shared memory the histogram needs (reserved in every mode so the walk and
// the scan run with the same launch shape, hence the same unit split).  Per
// bin: the sum of squared terms as a float scaled by 2^(-8(b-256)) (bin b
// holds bounds below 2^(4(b-256)+4), so a unit adds at most 2^(w+8)), and a
// 32-bit count; both have native shared-memory atomics.
constexpr size_t kHistSmemBytes = kHistBins * (sizeof(float) + sizeof(unsigned));
// Shared memory for the per-row bound terms (two per row, real or complex).
__host__ __device__ constexpr size_t bound_smem_bytes(int n) { return sizeof(double) * 2 * n; }

// 2^(4(b-256)) for bins 1..511 (bin 0 holds zero bounds, whose terms are 0),
// built from the exponent field; the histogram scale is its square.
__device__ __forceinline__ double hist_half_scale(int bin)
{
    const int b = bin < 1 ? 1 : bin;
    return __hiloint2double((1023 + 4 * (b - 256)) << 20, 0);
}
__device__ __forceinline__ double hist_half_unscale(int bin)
{
    const int b = bin < 1 ? 1 : bin;
    return __hiloint2double((1023 - 4 * (b - 256)) << 20, 0);
}

// Per-thread cache of the histogram: shared-memory atomics are issued only
// when a thread's bin changes from one unit to the next.
struct HistCache {
    int bin = -1;
    double s2 = 0.0;
    unsigned cnt = 0;
    __device__ __forceinline__ void add(int b, double v, float* s_hist, unsigned* s_cnt)
    {
        if (b != bin) {
            flush(s_hist, s_cnt);
            bin = b;
        }
        s2 += v;
        ++cnt;
    }
    __device__ __forceinline__ void flush(float* s_hist, unsigned* s_cnt)
    {
        if (cnt) {
            const double h = hist_half_unscale(bin);
            atomicAdd(&s_hist[bin], __double2float_rn((s2 * h) * h));
            atomicAdd(&s_cnt[bin], cnt);
        }
        s2 = 0.0;
        cnt = 0;
    }
};

// Flushes a CTA's shared histogram into the global one (double, 64-bit).
__device__ __forceinline__ void flush_hist(const float* s_hist, const unsigned* s_cnt, const Problem& pb)
{
    for (int i = threadIdx.x; i < kHistBins; i += blockDim.x)
        if (s_cnt[i]) {
            atomicAdd(&pb.hist_cnt[i], (unsigned long long)s_cnt[i]);
            const double h = hist_half_scale(i);
            atomicAdd(&pb.hist_s2[i], ((double)s_hist[i] * h) * h);
        }
}

// Thread caps keep the x vector (2 registers per double) plus the product
// chains under the per-thread register budget the cap implies
// (65536 / threads), so the walk never spills at the sizes that matter.
__host__ __device__ constexpr int RealMaxThreads(int n) { return n <= 40 ? 512 : 256; }
__host__ __device__ constexpr int ComplexMaxThreads(int n) { return n <= 10 ? 512 : (n <= 20 ? 384 : 256); }

template <int N>
struct RealCfg {
    static constexpr int G = N >= 3 ? 4 : (N == 2 ? 2 : 1);
    static constexpr int kMaxThreads = RealMaxThreads(N);
};

// Complex groups: four independent term chains per component while the
// x vector leaves room for them in registers (n <= 32), two beyond.
__host__ __device__ constexpr int ComplexGroup(int n) { return (n >= 3 && n <= 32) ? 4 : (n >= 2 ? 2 : 1); }

template <int N>
struct ComplexCfg {
    static constexpr int G = ComplexGroup(N);
    static constexpr int kMaxThreads = ComplexMaxThreads(N);
};

__device__ __forceinline__ dd ldcg_dd(const dd* p)
{
    return {__ldcg(&p->hi), __ldcg(&p->lo)};
}

// p[lane] + p[lane + 32] + ... over the entries below count, added in that
// order; the loads (through L2) are issued eight at a time ahead of the adds,
// so a lane waits for one round trip per eight entries, not one per entry.
__device__ __forceinline__ dd lane_sum_dd(const dd* p, int count, int lane)
{
    dd v = {0.0, 0.0};
    for (int b0 = lane; b0 < count; b0 += 32 * 8) {
        dd x[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = b0 + 32 * k < count ? ldcg_dd(p + b0 + 32 * k) : dd{0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (b0 + 32 * k < count) v = dd_add(v, x[k]);
    }
    return v;
}

// Warp -> block -> grid double-double reduction of C components.  The last
// CTA to finish (ticket election) sums the per-CTA partials in index order,
// so the result does not depend on CTA completion order.
template <int C>
__device__ __forceinline__ void grid_reduce(dd (&tot)[C], const Problem& pb)
{
    __shared__ dd s_warp[C][32];
    __shared__ int s_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int c = 0; c < C; ++c) tot[c] = warp_sum_dd(tot[c]);
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < C; ++c) s_warp[c][wid] = tot[c];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
            dd v = lane < nw ? s_warp[c][lane] : dd{0.0, 0.0};
            v = warp_sum_dd(v);
            if (lane == 0) pb.partials[c * pb.grid + blockIdx.x] = v;
        }
        if (lane == 0) {
            __threadfence();
            unsigned prev = atomicAdd(pb.ticket, 1u);
            s_last = (prev == gridDim.x - 1) ? 1 : 0;
        }
    }
    __syncthreads();
    if (s_last && wid == 0) {
        __threadfence();
#pragma unroll
        for (int c = 0; c < C; ++c) {
            dd v = lane_sum_dd(pb.partials + c * pb.grid, (int)gridDim.x, lane);
            v = warp_sum_dd(v);
            if (lane == 0) pb.result[c] = v;
        }
        if (lane == 0) *pb.ticket = 0u;
    }
}

// ---------------------------------------------------------------- real ----
// Sum over one unit: sum_d (-1)^popc(d) prod_r (xh_r + DE[d][r]).
// With STATS, also returns sum_d term_d^2 in *s2 (one FMA per term; sizes the
// double-double refinement).
template <int N, int G, bool STATS = false>
__device__ __forceinline__ double unit_sum_real(const double (&xh)[N], const double* __restrict__ s_de,
                                                int nq, double* s2 = nullptr)
{
    double acc = 0.0, sq[G];
#pragma unroll
    for (int i = 0; i < G; ++i) sq[i] = 0.0;
#pragma unroll 1
    for (int q = 0; q < nq; ++q) {
        const double* de = s_de + q * (N * G);
        double p[G];
        if constexpr (G == 4) {
            double2 v0 = reinterpret_cast<const double2*>(de)[0];
            double2 v1 = reinterpret_cast<const double2*>(de)[1];
            p[0] = add_rn(xh[0], v0.x);
            p[1] = add_rn(xh[0], v0.y);
            p[2] = add_rn(xh[0], v1.x);
            p[3] = add_rn(xh[0], v1.y);
#pragma unroll
            for (int r = 1; r < N; ++r) {
                double2 a = reinterpret_cast<const double2*>(de + r * 4)[0];
                double2 b = reinterpret_cast<const double2*>(de + r * 4)[1];
                p[0] = mul_rn(p[0], add_rn(xh[r], a.x));
                p[1] = mul_rn(p[1], add_rn(xh[r], a.y));
                p[2] = mul_rn(p[2], add_rn(xh[r], b.x));
                p[3] = mul_rn(p[3], add_rn(xh[r], b.y));
            }
        } else {
#pragma unroll
            for (int i = 0; i < G; ++i) p[i] = add_rn(xh[0], de[i]);
#pragma unroll
            for (int r = 1; r < N; ++r) {
#pragma unroll
                for (int i = 0; i < G; ++i) p[i] = mul_rn(p[i], add_rn(xh[r], de[r * G + i]));
            }
        }
        double gs;
        if constexpr (G == 4) gs = sub_rn(sub_rn(p[0], p[1]), sub_rn(p[2], p[3]));  // + - - +
        else if constexpr (G == 2) gs = sub_rn(p[0], p[1]);
        else gs = p[0];
        acc = (__popc(q) & 1) ? sub_rn(acc, gs) : add_rn(acc, gs);
        if constexpr (STATS) {
#pragma unroll
            for (int i = 0; i < G; ++i) sq[i] = __fma_rn(p[i], p[i], sq[i]);
        }
    }
    if constexpr (STATS) {
        double t = 0.0;
#pragma unroll
        for (int i = 0; i < G; ++i) t += sq[i];
        *s2 = t;
    }
    return acc;
}

// First unit base of each thread, built cooperatively by its warp from the
// NW start vector (x0h, x0l) and the high columns s_mt; every lane of the
// warp calls this (it shuffles), whether it owns units or not.
// The lanes' first units u0 lie in one range [ulo, uhi] (balanced_range is
// monotonic in the thread index), so the Gray bits above P, the highest bit
// where ulo and uhi differ, are the same for every lane.  Lane r adds the
// high columns j > P selected by those common bits to x0_r (double-double,
// ascending j) for rows r and r + 32, the warp broadcasts the N results,
// and each lane adds its own columns j <= P (ascending), four rows at a time
// (independent chains, the same operations per row).  Hi words go to xh,
// lo words to the thread's shared slots s_lo[r * bd + tid].  Compared with
// every lane adding all of its columns, this saves most of the double-double
// adds when threads own few units (n <= 26).
template <int N>
__device__ __forceinline__ void first_base_real(const double* __restrict__ x0h, const double* __restrict__ x0l,
                                                const double* __restrict__ s_mt, double* s_lo, int ntop,
                                                unsigned long long u0, unsigned long long u1, int tid, int bd,
                                                double (&xh)[N])
{
    const unsigned full = 0xffffffffu;
    const int lane = tid & 31;
    const unsigned act = __ballot_sync(full, u0 < u1);
    if (act == 0u) return;  // warp-uniform
    const int last = 31 - __clz(act);
    const unsigned long long ulo = __shfl_sync(full, u0, 0), uhi = __shfl_sync(full, u0, last);
    const int P = ulo == uhi ? -1 : 63 - __clzll(ulo ^ uhi);
    const unsigned long long gc = gray_of(ulo);
    dd c0 = {0.0, 0.0}, c1 = {0.0, 0.0};
    if (lane < N) {
        c0 = dd{x0h[lane], x0l[lane]};
        if (N > 32 && lane + 32 < N) c1 = dd{x0h[lane + 32], x0l[lane + 32]};
        for (int j = P + 1; j < ntop; ++j)
            if ((gc >> j) & 1ull) {
                c0 = dd_add_d(c0, s_mt[j * N + lane]);
                if (N > 32 && lane + 32 < N) c1 = dd_add_d(c1, s_mt[j * N + lane + 32]);
            }
    }
    const bool own = u0 < u1;
#pragma unroll
    for (int r = 0; r < N; ++r) {
        const double h = __shfl_sync(full, r < 32 ? c0.hi : c1.hi, r & 31);
        const double l = __shfl_sync(full, r < 32 ? c0.lo : c1.lo, r & 31);
        xh[r] = h;
        if (own) s_lo[r * bd + tid] = l;
    }
    if (!own) return;
    const unsigned long long g0 = gray_of(u0);
    const int jp = P + 1 < ntop ? P + 1 : ntop;  // private columns 0 .. jp-1
#pragma unroll
    for (int r0 = 0; r0 < N; r0 += 4) {
        dd x[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (r0 + k < N) x[k] = dd{xh[r0 + k], s_lo[(r0 + k) * bd + tid]};
        for (int j = 0; j < jp; ++j)
            if ((g0 >> j) & 1ull) {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (r0 + k < N) x[k] = dd_add_d(x[k], s_mt[j * N + r0 + k]);
            }
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (r0 + k < N) {
                xh[r0 + k] = x[k].hi;
                s_lo[(r0 + k) * bd + tid] = x[k].lo;
            }
    }
}

template <int N>
__global__ void __launch_bounds__(RealCfg<N>::kMaxThreads, 1) walk_real(Problem pb)
{
    constexpr int G = RealCfg<N>::G;
    extern __shared__ __align__(16) double smem[];
    const int w = pb.w;
    const int terms = 1 << w;
    const int nq = terms / G;
    const int ntop = N - 1 - w;
    const int tid = threadIdx.x, bd = blockDim.x;
    double* s_de = smem;
    double* s_mt = s_de + terms * N;
    double* s_lo = s_mt + (ntop > 0 ? ntop : 0) * N;
    float* s_hist = reinterpret_cast<float*>(s_lo + N * bd);  // mode 1
    unsigned* s_cnt = reinterpret_cast<unsigned*>(s_hist + kHistBins);
    // DE range per row, [2][N] (min, max).  Two scalar loads per row: a paired
    // 16-byte load keeps more registers live and makes the n=32 walk spill.
    double* s_bnd = reinterpret_cast<double*>(s_cnt + kHistBins);
    for (int i = tid; i < terms * N; i += bd) s_de[i] = pb.de_hi[i];
    for (int i = tid; i < ntop * N; i += bd) s_mt[i] = pb.mt[i];
    const int mode = pb.mode;
    if (mode != 0)
        for (int i = tid; i < 2 * N; i += bd) s_bnd[i] = pb.bnd[i];
    if (mode == 1)
        for (int i = tid; i < kHistBins; i += bd) { s_hist[i] = 0.0f; s_cnt[i] = 0u; }
    __syncthreads();

    const unsigned long long T = (unsigned long long)gridDim.x * bd;
    const unsigned long long t = (unsigned long long)blockIdx.x * bd + tid;
    unsigned long long u0, u1;
    balanced_range(pb.units, T, t, &u0, &u1);
    // The scan only walks threads that own a unit at or above the threshold.
    if (mode == 2 && (int)pb.tmax[t] < pb.thr_bin) u1 = u0;
    dd tot[1] = {{0.0, 0.0}};
    HistCache hc;
    const int lbin = mode == 1 ? __ldcg(pb.list_bin) : 0;
    int bmax = 0;
    double xh[N];
    // First unit base: x0 plus the selected high columns, the warp's common
    // ones first (the refinement rebuilds bases in plain index order; the hi
    // words agree unless a row value lies within ~2^-100 of a rounding
    // midpoint, and then only that unit's correction carries one FP64 rounding).
    first_base_real<N>(pb.x0_hi, pb.x0_lo, s_mt, s_lo, ntop, u0, u1, tid, bd, xh);
    if (u0 < u1) {
        unsigned long long u = u0;
        while (true) {
            int b = 0;
            if (mode != 0) {
                // Upper bound of |term| over the unit: prod_r max |xh_r + DE[d][r]|;
                // the scan recomputes it bit for bit to select the same units.
                double ub = 1.0;
#pragma unroll
                for (int r = 0; r < N; ++r)
                    ub = mul_rn(ub, fmax(fabs(add_rn(xh[r], s_bnd[r])), fabs(add_rn(xh[r], s_bnd[N + r]))));
                b = hist_bin(ub);
                bmax = b > bmax ? b : bmax;
                if (mode == 2 && b >= pb.thr_bin) {
                    unsigned long long k = atomicAdd(pb.list_n, 1ull);
                    if (k < pb.list_cap) {
                        pb.list_u[k] = u;
                        double* dst = pb.list_x + k * (2 * N);
#pragma unroll
                        for (int r = 0; r < N; ++r) { dst[r] = xh[r]; dst[N + r] = s_lo[r * bd + tid]; }
                    }
                }
            }
            if (mode == 0) {
                double us = unit_sum_real<N, G>(xh, s_de, nq);
                tot[0] = dd_add_d(tot[0], (u & 1ull) ? -us : us);
            } else if (mode == 1) {
                double sq;
                double us = unit_sum_real<N, G, true>(xh, s_de, nq, &sq);
                tot[0] = dd_add_d(tot[0], (u & 1ull) ? -us : us);
                hc.add(b, sq, s_hist, s_cnt);  // actual sum of squared terms, keyed by the bound
                raw_list_add(pb, lbin, u, b);
            }
            if (++u >= u1) break;
            const int j = __ffsll((long long)u) - 1;
            const bool add = (gray_of(u) >> j) & 1ull;
            const double* col = s_mt + j * N;
#pragma unroll
            for (int r = 0; r < N; ++r) {
                double m = add ? col[r] : -col[r];
                dd s = two_sum(xh[r], m);
                dd z = fast_two_sum(s.hi, add_rn(s.lo, s_lo[r * bd + tid]));
                xh[r] = z.hi;
                s_lo[r * bd + tid] = z.lo;
            }
        }
    }
    if (mode == 1) {
        pb.tmax[t] = (unsigned short)bmax;
        hc.flush(s_hist, s_cnt);
        __syncthreads();
        flush_hist(s_hist, s_cnt, pb);
    }
    if (mode != 2) grid_reduce<1>(tot, pb);
}

// ------------------------------------------------------------- complex ----
template <int N, int G, bool STATS = false>
__device__ __forceinline__ void unit_sum_complex(const double (&xr)[N], const double (&xi)[N],
                                                 const double* __restrict__ s_de_re,
                                                 const double* __restrict__ s_de_im, int nq,
                                                 double& acc_re, double& acc_im, double* s2 = nullptr)
{
    double ar = 0.0, ai = 0.0, sq[G];
#pragma unroll
    for (int i = 0; i < G; ++i) sq[i] = 0.0;
#pragma unroll 1
    for (int q = 0; q < nq; ++q) {
        const double* dr = s_de_re + q * (N * G);
        const double* di = s_de_im + q * (N * G);
        double pr[G], pi[G];
#pragma unroll
        for (int i = 0; i < G; ++i) {
            pr[i] = add_rn(xr[0], dr[i]);
            pi[i] = add_rn(xi[0], di[i]);
        }
#pragma unroll
        for (int r = 1; r < N; ++r) {
            double vr[G], vi[G];
            if constexpr (G == 4) {
                double2 a0 = reinterpret_cast<const double2*>(dr + r * 4)[0];
                double2 a1 = reinterpret_cast<const double2*>(dr + r * 4)[1];
                double2 b0 = reinterpret_cast<const double2*>(di + r * 4)[0];
                double2 b1 = reinterpret_cast<const double2*>(di + r * 4)[1];
                vr[0] = a0.x; vr[1] = a0.y; vr[2] = a1.x; vr[3] = a1.y;
                vi[0] = b0.x; vi[1] = b0.y; vi[2] = b1.x; vi[3] = b1.y;
            } else if constexpr (G == 2) {
                double2 a = reinterpret_cast<const double2*>(dr + r * 2)[0];
                double2 b = reinterpret_cast<const double2*>(di + r * 2)[0];
                vr[0] = a.x; vr[1] = a.y; vi[0] = b.x; vi[1] = b.y;
            } else {
#pragma unroll
                for (int i = 0; i < G; ++i) { vr[i] = dr[r * G + i]; vi[i] = di[r * G + i]; }
            }
#pragma unroll
            for (int i = 0; i < G; ++i) {
                double yr = add_rn(xr[r], vr[i]);
                double yi = add_rn(xi[r], vi[i]);
                double t1 = mul_rn(pi[i], yi);
                double t2 = mul_rn(pi[i], yr);
                double nr = __fma_rn(pr[i], yr, -t1);
                double ni = __fma_rn(pr[i], yi, t2);
                pr[i] = nr;
                pi[i] = ni;
            }
        }
        double gr, gi;
        if constexpr (G == 4) {  // + - - +
            gr = sub_rn(sub_rn(pr[0], pr[1]), sub_rn(pr[2], pr[3]));
            gi = sub_rn(sub_rn(pi[0], pi[1]), sub_rn(pi[2], pi[3]));
        } else if constexpr (G == 2) { gr = sub_rn(pr[0], pr[1]); gi = sub_rn(pi[0], pi[1]); }
        else { gr = pr[0]; gi = pi[0]; }
        if (__popc(q) & 1) { ar = sub_rn(ar, gr); ai = sub_rn(ai, gi); }
        else { ar = add_rn(ar, gr); ai = add_rn(ai, gi); }
        if constexpr (STATS) {
#pragma unroll
            for (int i = 0; i < G; ++i) sq[i] = __fma_rn(pi[i], pi[i], __fma_rn(pr[i], pr[i], sq[i]));
        }
    }
    acc_re = ar;
    acc_im = ai;
    if constexpr (STATS) {
        double t = 0.0;
#pragma unroll
        for (int i = 0; i < G; ++i) t += sq[i];
        *s2 = t;
    }
}

template <int N>
__global__ void __launch_bounds__(ComplexCfg<N>::kMaxThreads, 1) walk_complex(Problem pb)
{
    constexpr int G = ComplexCfg<N>::G;
    extern __shared__ __align__(16) double smem[];
    const int w = pb.w;
    const int terms = 1 << w;
    const int nq = terms / G;
    const int ntop = N - 1 - w;
    const int ntp = ntop > 0 ? ntop : 0;
    const int tid = threadIdx.x, bd = blockDim.x;
    double* s_de = smem;                        // [2][terms*N]
    double* s_mt = s_de + 2 * terms * N;        // [2][ntop*N]
    double* s_lo = s_mt + 2 * ntp * N;          // [2][N][bd]
    float* s_hist = reinterpret_cast<float*>(s_lo + 2 * N * bd);  // mode 1
    unsigned* s_cnt = reinterpret_cast<unsigned*>(s_hist + kHistBins);
    double* s_bnd = reinterpret_cast<double*>(s_cnt + kHistBins);  // [N]
    for (int i = tid; i < 2 * terms * N; i += bd) s_de[i] = pb.de_hi[i];
    for (int i = tid; i < 2 * ntp * N; i += bd) s_mt[i] = pb.mt[i];
    const int mode = pb.mode;
    if (mode != 0)
        for (int i = tid; i < N; i += bd) s_bnd[i] = pb.bnd[i];
    if (mode == 1)
        for (int i = tid; i < kHistBins; i += bd) { s_hist[i] = 0.0f; s_cnt[i] = 0u; }
    __syncthreads();
    const double* s_mt_re = s_mt;
    const double* s_mt_im = s_mt + ntp * N;
    double* s_lo_re = s_lo;
    double* s_lo_im = s_lo + N * bd;

    const unsigned long long T = (unsigned long long)gridDim.x * bd;
    const unsigned long long t = (unsigned long long)blockIdx.x * bd + tid;
    unsigned long long u0, u1;
    balanced_range(pb.units, T, t, &u0, &u1);
    if (mode == 2 && (int)pb.tmax[t] < pb.thr_bin) u1 = u0;
    dd tot[2] = {{0.0, 0.0}, {0.0, 0.0}};
    HistCache hc;
    const int lbin = mode == 1 ? __ldcg(pb.list_bin) : 0;
    int bmax = 0;
    if (u0 < u1) {
        double xr[N], xi[N];
        const unsigned long long g0 = gray_of(u0);
        // Two rows (four add chains) at a time, the same operations per row.
#pragma unroll
        for (int r0 = 0; r0 < N; r0 += 2) {
            dd a[2], b[2];
#pragma unroll
            for (int k = 0; k < 2; ++k)
                if (r0 + k < N) {
                    a[k] = dd{pb.x0_hi[r0 + k], pb.x0_lo[r0 + k]};
                    b[k] = dd{pb.x0_hi[N + r0 + k], pb.x0_lo[N + r0 + k]};
                }
            for (int j = 0; j < ntop; ++j)
                if ((g0 >> j) & 1ull) {
#pragma unroll
                    for (int k = 0; k < 2; ++k)
                        if (r0 + k < N) {
                            a[k] = dd_add_d(a[k], s_mt_re[j * N + r0 + k]);
                            b[k] = dd_add_d(b[k], s_mt_im[j * N + r0 + k]);
                        }
                }
#pragma unroll
            for (int k = 0; k < 2; ++k)
                if (r0 + k < N) {
                    xr[r0 + k] = a[k].hi;
                    xi[r0 + k] = b[k].hi;
                    s_lo_re[(r0 + k) * bd + tid] = a[k].lo;
                    s_lo_im[(r0 + k) * bd + tid] = b[k].lo;
                }
        }
        unsigned long long u = u0;
        while (true) {
            int b = 0;
            if (mode != 0) {
                // |x_r| <= |xtop_r| + max_d |DE[d][r]|  (triangle inequality)
                double ub = 1.0;
#pragma unroll
                for (int r = 0; r < N; ++r)
                    ub = mul_rn(ub, add_rn(__dsqrt_rn(__fma_rn(xr[r], xr[r], mul_rn(xi[r], xi[r]))), s_bnd[r]));
                b = hist_bin(ub);
                bmax = b > bmax ? b : bmax;
                if (mode == 2 && b >= pb.thr_bin) {
                    unsigned long long k = atomicAdd(pb.list_n, 1ull);
                    if (k < pb.list_cap) {
                        pb.list_u[k] = u;
                        double* dst = pb.list_x + k * (4 * N);
#pragma unroll
                        for (int r = 0; r < N; ++r) {
                            dst[r] = xr[r];
                            dst[N + r] = s_lo_re[r * bd + tid];
                            dst[2 * N + r] = xi[r];
                            dst[3 * N + r] = s_lo_im[r * bd + tid];
                        }
                    }
                }
            }
            if (mode != 2) {
                double ur, ui, sq = 0.0;
                if (mode == 0) unit_sum_complex<N, G>(xr, xi, s_de, s_de + terms * N, nq, ur, ui);
                else unit_sum_complex<N, G, true>(xr, xi, s_de, s_de + terms * N, nq, ur, ui, &sq);
                if (u & 1ull) { ur = -ur; ui = -ui; }
                tot[0] = dd_add_d(tot[0], ur);
                tot[1] = dd_add_d(tot[1], ui);
                if (mode == 1) {
                    hc.add(b, sq, s_hist, s_cnt);
                    raw_list_add(pb, lbin, u, b);
                }
            }
            if (++u >= u1) break;
            const int j = __ffsll((long long)u) - 1;
            const bool add = (gray_of(u) >> j) & 1ull;
#pragma unroll
            for (int r = 0; r < N; ++r) {
                double mr = add ? s_mt_re[j * N + r] : -s_mt_re[j * N + r];
                double mi = add ? s_mt_im[j * N + r] : -s_mt_im[j * N + r];
                dd s = two_sum(xr[r], mr);
                dd z = fast_two_sum(s.hi, add_rn(s.lo, s_lo_re[r * bd + tid]));
                xr[r] = z.hi;
                s_lo_re[r * bd + tid] = z.lo;
                s = two_sum(xi[r], mi);
                z = fast_two_sum(s.hi, add_rn(s.lo, s_lo_im[r * bd + tid]));
                xi[r] = z.hi;
                s_lo_im[r * bd + tid] = z.lo;
            }
        }
    }
    if (mode == 1) {
        pb.tmax[t] = (unsigned short)bmax;
        hc.flush(s_hist, s_cnt);
        __syncthreads();
        flush_hist(s_hist, s_cnt, pb);
    }
    if (mode != 2) grid_reduce<2>(tot, pb);
}

// Double-double refinement (dense_refine.cu), all stream-ordered after the
// mode-1 walk with no host round trip in between:
//   launch_threshold   picks rb->thr / rb->count / rb->err from the
//                      histogram and decides the listing path (rb->from_list);
//   launch_listing     lists the units whose bin >= rb->thr: from the walk's
//                      own list when rb->from_list, else from the walk's
//                      per-thread maxima (pb.tmax), one warp per thread
//                      range, bases rebuilt from scratch;
//   launch_refine      re-evaluates the listed units in double-double and
//                      writes sum(double-double unit sum - the walk's FP64
//                      unit sum) to rb->corr, a worker of one or more warps
//                      per unit; it refines nothing unless
//                      rb->list_n == rb->count <= pb.list_cap.
// bound_walk + pick_list_bin run before the walk and set the bin from which
// the walk lists its units.  A mode-2 walk (same launch shape as mode 1)
// replays the listing with the walk's own bases (pb.list_x) when the host
// finds the count check failed.
int launch_threshold(const Problem& pb, cudaStream_t s);
int launch_refine(const Problem& pb, int blocks, cudaStream_t s);
int launch_bound_pass(const Problem& pb, int blocks, cudaStream_t s);
int launch_listing(const Problem& pb, cudaStream_t s);
// Dynamic shared memory of the refinement at `threads` threads per CTA: both
// words of every part's table, per-warp bases and group sums, high columns.
size_t refine_smem_bytes(const Problem& pb, int threads);

// FP32-product walks (f32_impl.cuh), n <= kMaxF32N.  A result whose
// estimated relative error exceeds opt.rel_tol (kF32DefaultBound when unset,
// the library's accuracy bar) comes back with SPB_ERR_ACCURACY.
constexpr int kMaxF32N = 40;
constexpr double kF32DefaultBound = 1e-12;
int launch_walk_f32(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s);
size_t walk_f32_smem_bytes(const Problem& pb, int threads);
int walk_f32_max_threads(int n, int comps);

// Per-n dispatch (defined in the instantiation units).
int launch_walk_real(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s);
int launch_walk_complex(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s);

// Row-compacted walk on NA = pb.na active rows (sparse_walk.cu).
int launch_walk_sparse(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s);

inline int launch_walk(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s)
{
    if (pb.na < pb.n) return launch_walk_sparse(pb, blocks, threads, smem, s);
    return pb.comps == 1 ? launch_walk_real(pb, blocks, threads, smem, s)
                         : launch_walk_complex(pb, blocks, threads, smem, s);
}

int walk_max_threads(int n, int comps);

}  // namespace dense
}  // namespace spb

// X-macro over n = 1..63.
#define SPB_FOR_EACH_N(X)                                                                  \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15)       \
    X(16) X(17) X(18) X(19) X(20) X(21) X(22) X(23) X(24) X(25) X(26) X(27) X(28) X(29)    \
    X(30) X(31) X(32) X(33) X(34) X(35) X(36) X(37) X(38) X(39) X(40) X(41) X(42) X(43)    \
    X(44) X(45) X(46) X(47) X(48) X(49) X(50) X(51) X(52) X(53) X(54) X(55) X(56) X(57)    \
    X(58) X(59) X(60) X(61) X(62) X(63)
