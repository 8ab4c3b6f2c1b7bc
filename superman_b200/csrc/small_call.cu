// One cooperative kernel for a whole dense real permanent of small size
// (4 <= n <= kSmallCallMaxN), in FP64 mode or with the double-double
// refinement.
//
// At these sizes the Gray walk itself is a few tens of microseconds, and a
// call made of separate kernels (setup, walk, threshold, listing, refinement)
// spends about as long again in launches, one-CTA phases and the gaps between
// kernels.  Here every CTA of a persistent grid (one per SM, launched
// cooperatively so that all are resident) does the whole call:
//   0. builds the tables the walk reads in its own shared memory from the
//      matrix: row scaling by powers of two, the double-double NW start vector
//      and subset-sum table, the high columns and the per-row bound ranges,
//      with the operations of setup_kernel, so the values are the same;
//      CTA 0 also zeroes the call's global accumulators; grid barrier;
//   1. evaluates the units in passes over the grid (thread t owns units t,
//      t + T, ...; with no more units than the T threads of the grid, unit t
//      alone, the split walk_real makes then) with walk_real's evaluators,
//      on unit bases its warp builds row-parallel
//      (double-double, so their hi words are walk_real's but for values
//      within ~2^-104 of a rounding midpoint), binning each unit by its
//      bound and recording the bin per unit; CTA totals go to pb.partials;
//      grid barrier;
//   2. every CTA sums the CTA totals in index order (the grid total, as
//      grid_reduce forms it) and, with the refinement, picks the threshold
//      from the histogram (staged in shared memory; one warp,
//      pick_threshold_shared);
//   3. with the refinement, each thread lists its units at or above the
//      threshold; grid barrier; the listed units are dealt out one per CTA
//      and re-evaluated by the whole CTA in double-double (base rebuilt from
//      x0 and the high columns, as refine_real does), against the FP64 value
//      the walk stored for the unit; the last CTA sums the corrections in
//      index order.
// The last CTA to finish copies the readback into page-locked host memory
// mapped into the device's address space, so the host copies nothing after
// the kernel.  Nothing waits on anything but the grid barriers of
// cooperative groups.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "context.h"
#include "dense_impl.cuh"
#include "refine_impl.cuh"

namespace cg = cooperative_groups;

namespace spb {
namespace dense {

constexpr int kSmallCallMaxN = 26;
constexpr int kSmallCallThreads = 512;

namespace {

__host__ __device__ constexpr size_t even(size_t v) { return (v + 1) & ~(size_t)1; }

// Shared-memory layout, in doubles from the dynamic base; every array
// starts 16-byte aligned (the evaluators read the table with 16-byte loads).
struct SmallLayout {
    size_t a, x0h, x0l, dh, dl, mt, base, bnd, xw, hist, total;
    __host__ __device__ SmallLayout(int n, int w, int threads)
    {
        const size_t terms = (size_t)1 << w, ntop = n - 1 - w > 0 ? n - 1 - w : 0;
        const size_t warps = threads / 32;
        a = 0;
        x0h = even(a + (size_t)n * n);
        x0l = even(x0h + n);
        dh = even(x0l + n);
        dl = even(dh + terms * n);
        mt = even(dl + terms * n);
        // [warps][n][33] the walk's unit bases (hi words); after the walk, the
        // staged histogram (2 x kHistPadded doubles)
        base = even(mt + ntop * n);
        const size_t nb = warps * (size_t)n * 33 > 2 * (size_t)kHistPadded ? warps * (size_t)n * 33
                                                                           : 2 * (size_t)kHistPadded;
        bnd = even(base + nb);
        xw = even(bnd + 2 * (size_t)n);          // [2n] the refined unit's base, hi then lo
        hist = even(xw + 2 * (size_t)n);          // float[kHistBins] + unsigned[kHistBins]
        total = hist + (kHistSmemBytes + sizeof(double) - 1) / sizeof(double);
    }
    size_t bytes() const { return total * sizeof(double); }
};

// Sum over the CTA in warp order; valid in thread 0.
__device__ __forceinline__ dd block_sum_dd(dd v, dd* s_warp)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum_dd(v);
    if (lane == 0) s_warp[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < nw ? s_warp[lane] : dd{0.0, 0.0};
        v = warp_sum_dd(v);
    }
    __syncthreads();
    return v;
}

// Copies the finished readback to the host's page-locked copy (mapped into
// the device's address space), reading it through L2: its fields were
// written by other CTAs.  The host then needs no copy after the kernel.
__device__ __forceinline__ void publish(const Problem& pb, Readback* host)
{
    if (!host) return;
    __threadfence();
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(pb.rb);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(host);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(Readback) / sizeof(unsigned long long)); ++i) dst[i] = __ldcg(src + i);
}
static_assert(sizeof(Readback) % sizeof(unsigned long long) == 0, "readback copied in 8-byte words");

// The walk's FP64 value of each unit, kept for the refinement in the space
// of the separate kernels' unit list (pb.raw_u, kRawCap entries of 8 bytes,
// unused by this call; units <= kRawCap here).
__device__ __forceinline__ double* unit_value(const Problem& pb) { return reinterpret_cast<double*>(pb.raw_u); }

template <int N>
__global__ void __launch_bounds__(kSmallCallThreads, 1) small_call_real(Problem pb, const double* a_in,
                                                                         const double* a_stage, Readback* rb_host)
{
    constexpr int G = RealCfg<N>::G;
    cg::grid_group grid = cg::this_grid();
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_exp[N];
    __shared__ dd s_warp[32];
    __shared__ dd s_total;
    __shared__ int s_thr;
    __shared__ unsigned long long s_count;
    __shared__ double s_err;
    __shared__ int s_last;
    const int w = pb.w, terms = 1 << w, nq = terms / G, ntop = N - 1 - w;
    const int tid = threadIdx.x, bd = blockDim.x, lane = tid & 31, wid = tid >> 5;
    const int mode = pb.mode;
    const SmallLayout L(N, w, bd);
    double* s_a = smem + L.a;
    double* s_x0h = smem + L.x0h;
    double* s_x0l = smem + L.x0l;
    double* s_dh = smem + L.dh;
    double* s_dl = smem + L.dl;
    double* s_mt = smem + L.mt;
    double* s_bnd = smem + L.bnd;
    float* s_hist = reinterpret_cast<float*>(smem + L.hist);
    unsigned* s_cnt = reinterpret_cast<unsigned*>(s_hist + kHistBins);

    // ---- 0. the zeroed accumulators and the tables (setup_kernel's
    // operations).  A host matrix arrives staged in page-locked memory
    // (a_stage, mapped): the grid copies it to a_in first, one element per
    // thread, and meets at a barrier, which also publishes the zeroed
    // accumulators; a device matrix is read where it is.
    const bool staged = a_stage != nullptr;  // the same in every CTA
    if (blockIdx.x == 0) {
        if (tid < 4) pb.ticket[tid] = 0u;
        if (mode != 0)
            for (int i = tid; i < kHistBins; i += bd) {
                pb.hist_s2[i] = 0.0;
                pb.hist_cnt[i] = 0ull;
            }
        if (tid == 0) *pb.list_n = 0ull;
    }
    if (staged) {
        double* a_dev = const_cast<double*>(a_in);
        for (int i = blockIdx.x * bd + tid; i < N * N; i += gridDim.x * bd) a_dev[i] = a_stage[i];
        grid.sync();
        for (int i = tid; i < N * N; i += bd) s_a[i] = __ldcg(a_in + i);
    } else {
        for (int i = tid; i < N * N; i += bd) s_a[i] = a_in[i];
    }
    if (mode != 0)
        for (int i = tid; i < kHistBins; i += bd) { s_hist[i] = 0.0f; s_cnt[i] = 0u; }
    __syncthreads();
    // row maxima of |a|, a warp per row (fmax does not depend on the order)
    static_assert(N <= 32, "a row fits a warp");
    for (int r = wid; r < N; r += bd / 32) {
        double mx = lane < N ? fabs(s_a[r * N + lane]) : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        if (lane == 0) {
            int e = 0;
            if (mx > 0.0 && isfinite(mx)) frexp(mx, &e);
            s_exp[r] = e;
        }
    }
    __syncthreads();
    for (int i = tid; i < N * N; i += bd) s_a[i] = ldexp(s_a[i], -s_exp[i / N]);
    __syncthreads();
    // The NW start vector x0 (one row per lane of the CTA's last warp, n
    // dependent adds each) and the subset-sum table (the other warps, a row
    // each at a time) are built side by side.  A row's table is built level
    // by level, DE[d][r] = DE[d - 2^k][r] + a_rk for d in [2^k, 2^(k+1)),
    // its lanes taking a level's entries and meeting at a warp barrier; the
    // values are setup_kernel's.  Layout [d/G][r][d%G].
    auto pos = [&](int d, int r) { return ((d / G) * N + r) * G + (d % G); };
    const int nw = bd >> 5;
    const int xwarp = nw > 1 ? nw - 1 : 0;  // the x0 warp
    if (wid == xwarp && lane < N) {
        const int r = lane;
        dd s = {0.0, 0.0};
        for (int j = 0; j < N; ++j) s = dd_add_d(s, s_a[r * N + j]);
        dd h = {-0.5 * s.hi, -0.5 * s.lo};  // exact halving
        dd x = dd_add_d(h, s_a[r * N + (N - 1)]);
        s_x0h[r] = x.hi;
        s_x0l[r] = x.lo;
    }
    if (blockIdx.x == 0 && tid == bd - 1) {  // lane 31 of the x0 warp: not a row thread (N < 32)
        int es = 0;
        for (int r = 0; r < N; ++r) es += s_exp[r];
        *pb.exp_sum = es;
    }
    const int tw = nw > 1 ? nw - 1 : 1;  // warps building the table
    if (wid < tw)
        for (int r0 = wid; r0 < N; r0 += 2 * tw) {
            // two rows side by side (independent chains); r1 may be past n
            const int r1 = r0 + tw;
            const bool two = r1 < N;
            if (lane == 0) {
                s_dh[pos(0, r0)] = 0.0;
                s_dl[pos(0, r0)] = 0.0;
                if (two) {
                    s_dh[pos(0, r1)] = 0.0;
                    s_dl[pos(0, r1)] = 0.0;
                }
            }
            for (int k = 0; k < w; ++k) {
                __syncwarp();
                const int half = 1 << k;
                const double a0 = s_a[r0 * N + k], a1 = two ? s_a[r1 * N + k] : 0.0;
                for (int e = lane; e < half; e += 32) {
                    const dd v0 = dd_add_d(dd{s_dh[pos(e, r0)], s_dl[pos(e, r0)]}, a0);
                    if (two) {
                        const dd v1 = dd_add_d(dd{s_dh[pos(e, r1)], s_dl[pos(e, r1)]}, a1);
                        s_dh[pos(half + e, r1)] = v1.hi;
                        s_dl[pos(half + e, r1)] = v1.lo;
                    }
                    s_dh[pos(half + e, r0)] = v0.hi;
                    s_dl[pos(half + e, r0)] = v0.lo;
                }
            }
            __syncwarp();
        }
    if (mode != 0)
        for (int r = tid; r < N; r += bd) {
            double lo = 0.0, hi = 0.0;
            for (int j = 0; j < w; ++j) {
                const double v = s_a[r * N + j];
                if (v < 0.0) lo += v; else hi += v;
            }
            s_bnd[r] = lo;
            s_bnd[N + r] = hi;
        }
    for (int idx = tid; idx < ntop * N; idx += bd) {
        const int j = idx / N, r = idx % N;
        s_mt[idx] = s_a[r * N + (w + j)];
    }
    __syncthreads();
    if (!staged) grid.sync();  // the zeroed accumulators are visible before anyone adds to them

    // ---- 1. the walk, one unit per thread and pass, evaluated as walk_real
    // evaluates it.  In each pass the warp builds its 32 unit bases
    // row-parallel: lane r adds the selected high columns of the
    // warp's first unit to x0_r in ascending order (double-double, as the
    // refinement rebuilds a base), then takes the 31 Gray steps to the
    // following units with walk_real's double-double step, storing each hi
    // word; each lane then reads its own unit's row values.  That is 16 adds
    // plus 31 steps per row and warp, where building each lane's base alone
    // costs every lane its own adds for all rows.
    // With more units than threads the grid takes them in passes: thread t
    // owns units t, t + T, t + 2T, ... (T threads in the grid).
    const unsigned long long T = (unsigned long long)gridDim.x * bd;
    const unsigned long long t0 = (unsigned long long)blockIdx.x * bd + tid;
    double* s_base = smem + L.base + (size_t)wid * N * 33;  // [N][33]
    dd tot = {0.0, 0.0};
    int bin0 = -1, bin1 = -1;  // this thread's bins in the first two passes (listing reads the rest back)
    for (unsigned long long u = t0;; u += T) {
        const unsigned long long ub = u - (unsigned long long)lane;  // the warp's first unit
        if (ub >= pb.units) break;  // the same in every lane of the warp
        __syncwarp();               // the previous pass's bases are read
        if (lane < N) {
            const int r = lane;
            const unsigned long long g = gray_of(ub);
            dd x = {s_x0h[r], s_x0l[r]};
            for (int j = 0; j < ntop; ++j)
                if ((g >> j) & 1ull) x = dd_add_d(x, s_mt[j * N + r]);
            s_base[r * 33] = x.hi;
            for (int k = 1; k < 32 && ub + k < pb.units; ++k) {
                const unsigned long long v = ub + k;
                const int j = __ffsll((long long)v) - 1;
                const double c = s_mt[j * N + r];
                const dd sm = two_sum(x.hi, ((gray_of(v) >> j) & 1ull) ? c : -c);
                x = fast_two_sum(sm.hi, add_rn(sm.lo, x.lo));
                s_base[r * 33 + k] = x.hi;
            }
        }
        __syncwarp();
        int b = -1;  // this lane's histogram bin in this pass (-1: no unit)
        double sq = 0.0;
        if (u < pb.units) {
            double xh[N];
#pragma unroll
            for (int r = 0; r < N; ++r) xh[r] = s_base[r * 33 + lane];
            if (mode == 0) {
                const double us = unit_sum_real<N, G>(xh, s_dh, nq);
                tot = dd_add_d(tot, (u & 1ull) ? -us : us);
            } else {
                double ubd = 1.0;
#pragma unroll
                for (int r = 0; r < N; ++r)
                    ubd = mul_rn(ubd, fmax(fabs(add_rn(xh[r], s_bnd[r])), fabs(add_rn(xh[r], s_bnd[N + r]))));
                b = hist_bin(ubd);
                pb.raw_b[u] = (unsigned short)b;
                if (u == t0) bin0 = b;
                else if (u == t0 + T) bin1 = b;
                const double us = unit_sum_real<N, G, true>(xh, s_dh, nq, &sq);
                tot = dd_add_d(tot, (u & 1ull) ? -us : us);
                unit_value(pb)[u] = us;  // what the refinement corrects
            }
        }
        if (mode != 0) {
            // Neighbouring units share bins, so the lanes of a warp with the
            // same bin are summed by shuffles first and one shared atomic per
            // bin and warp is issued.
            const unsigned full = 0xffffffffu;
            float v = 0.0f;
            if (b >= 0) {
                const double h = hist_half_unscale(b);
                v = __double2float_rn((sq * h) * h);
            }
            unsigned pending = __ballot_sync(full, b >= 0);
            while (pending) {
                const int leader = __ffs(pending) - 1;
                const int lb = __shfl_sync(full, b, leader);
                const bool mine = b == lb;
                float x = mine ? v : 0.0f;
                unsigned c = mine ? 1u : 0u;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    x += __shfl_xor_sync(full, x, off);
                    c += __shfl_xor_sync(full, c, off);
                }
                if (lane == leader) {
                    atomicAdd(&s_hist[lb], x);
                    atomicAdd(&s_cnt[lb], c);
                }
                pending &= ~__ballot_sync(full, mine);
            }
        }
    }
    if (mode != 0) {
        __syncthreads();
        flush_hist(s_hist, s_cnt, pb);
    }
    // CTA total, reduced as grid_reduce does
    const dd cta = block_sum_dd(tot, s_warp);
    if (tid == 0) pb.partials[blockIdx.x] = cta;
    grid.sync();

    // ---- 2. grid total (index order, every CTA alike) and the threshold.
    // The whole CTA first copies the histogram into shared memory (the unit
    // bases' space, free now) with coalesced loads: read directly, each
    // lane's 16 consecutive bins cost one L2 request per bin.
    double* s_h2 = smem + L.base;
    unsigned long long* s_hc = reinterpret_cast<unsigned long long*>(s_h2 + kHistPadded);
    dd v = {0.0, 0.0};
    if (wid == 0) v = lane_sum_dd(pb.partials, (int)gridDim.x, lane);  // its loads overlap the staging
    if (mode != 0) {
        for (int b = tid; b < kHistBins; b += bd) {
            s_h2[hist_pad_index(b)] = __ldcg(pb.hist_s2 + b);
            s_hc[hist_pad_index(b)] = __ldcg(pb.hist_cnt + b);
        }
        __syncthreads();
    }
    if (wid == 0) {
        v = warp_sum_dd(v);
        if (lane == 0) s_total = v;
        if (mode != 0) {
            const double mag = fabs(v.hi);
            const ThresholdPick pk = pick_threshold_shared(pb, mag, s_h2, s_hc);
            if (lane == 0) {
                s_thr = pk.thr;
                s_count = pk.count;
                s_err = pk.err;
            }
        }
    }
    __syncthreads();
    if (blockIdx.x == 0 && tid == 0) {
        pb.rb->res[0] = s_total;
        pb.rb->corr[0] = dd{0.0, 0.0};
        if (mode != 0) {
            pb.rb->thr = s_thr;
            pb.rb->count = s_count;
            pb.rb->err = s_err;
            pb.rb->from_list = 1;
        }
        if (mode == 0 || s_thr >= kHistBins) publish(pb, rb_host);
    }
    if (mode == 0 || s_thr >= kHistBins) return;  // nothing to refine (uniform over the grid)

    // ---- 3. refinement of the units at or above the threshold.  Each thread
    // lists its units that qualify; after a grid barrier the listed units
    // are dealt out one per CTA in list order, so a cluster of dominant units
    // (they gather near the empty and the full subsets) spreads over the grid,
    // and each is refined by a whole CTA.
    const int thr = s_thr;
    for (unsigned long long u = t0; u < pb.units; u += T) {
        const int b = u == t0 ? bin0 : (u == t0 + T ? bin1 : (int)pb.raw_b[u]);
        if (b >= thr) {
            const unsigned long long k = atomicAdd(pb.list_n, 1ull);
            if (k < pb.list_cap) pb.list_u[k] = u;
        }
    }
    grid.sync();
    const unsigned long long listed = __ldcg(pb.list_n);
    const unsigned long long nl = listed < pb.list_cap ? listed : 0ull;  // overflow: the host falls back
    double* xw = smem + L.xw;  // [2N]: the unit base, hi then lo
    // threads per term: a power of two up to a warp (so a term's threads are
    // lanes of one warp and every warp's terms are all in range or all out),
    // as many as the CTA holds for all terms at once; each takes a run of rows
    int per = 1;
    while (per < 32 && 2 * per * terms <= bd) per *= 2;
    const int sub = tid % per, r0 = sub * N / per, r1 = (sub + 1) * N / per;
    dd corr = {0.0, 0.0};
    for (unsigned long long k = blockIdx.x; k < nl; k += gridDim.x) {
        const unsigned long long u = __ldcg(pb.list_u + k);
        const double walked = __ldcg(unit_value(pb) + u);  // in flight during the rebuild
        const unsigned long long g = gray_of(u);
        // unit base rebuilt from scratch in double-double (x0 plus the
        // selected high columns in index order), as refine_real does
        for (int r = tid; r < N; r += bd) {
            dd x = {s_x0h[r], s_x0l[r]};
            for (int j = 0; j < ntop; ++j)
                if ((g >> j) & 1ull) x = dd_add_d(x, s_mt[j * N + r]);
            xw[r] = x.hi;
            xw[N + r] = x.lo;
        }
        __syncthreads();
        // its double-double value: each term's product over the rows of
        // `per` threads, joined by shuffles
        dd acc = {0.0, 0.0};
        for (int d = tid / per; d < terms; d += bd / per) {
            dd p = {1.0, 0.0};
            for (int r = r0; r < r1; ++r)
                p = dd_mul(p, dd_add_fast(dd{xw[r], xw[N + r]}, dd{s_dh[pos(d, r)], s_dl[pos(d, r)]}));
            for (int off = 1; off < per; off <<= 1) p = dd_mul(p, shfl_xor_dd(p, off));
            if (sub == 0) acc = (__popc(d) & 1) ? dd_add(acc, dd_neg(p)) : dd_add(acc, p);
        }
        acc = block_sum_dd(acc, s_warp);
        if (tid == 0) {
            // against the value the walk added for this unit
            dd c = dd_add_d(acc, -walked);
            if (u & 1ull) c = dd_neg(c);
            corr = dd_add(corr, c);
        }
        __syncthreads();  // xw is rewritten by the next unit
    }
    if (tid == 0) {
        pb.partials[gridDim.x + blockIdx.x] = corr;
        __threadfence();
        const unsigned prev = atomicAdd(pb.ticket, 1u);
        s_last = prev == gridDim.x - 1 ? 1 : 0;
    }
    __syncthreads();
    if (s_last && wid == 0) {
        __threadfence();
        dd v = lane_sum_dd(pb.partials + gridDim.x, (int)gridDim.x, lane);
        v = warp_sum_dd(v);
        if (lane == 0) {
            pb.rb->corr[0] = v;
            *pb.ticket = 0u;
            publish(pb, rb_host);
        }
    }
}

using SmallKernel = void (*)(Problem, const double*, const double*, Readback*);

SmallKernel small_kernel(int n)
{
    switch (n) {
#define SPB_SCASE(N) \
    case N: return small_call_real<N>;
        SPB_SCASE(4) SPB_SCASE(5) SPB_SCASE(6) SPB_SCASE(7) SPB_SCASE(8) SPB_SCASE(9) SPB_SCASE(10)
        SPB_SCASE(11) SPB_SCASE(12) SPB_SCASE(13) SPB_SCASE(14) SPB_SCASE(15) SPB_SCASE(16)
        SPB_SCASE(17) SPB_SCASE(18) SPB_SCASE(19) SPB_SCASE(20) SPB_SCASE(21) SPB_SCASE(22)
        SPB_SCASE(23) SPB_SCASE(24) SPB_SCASE(25) SPB_SCASE(26)
#undef SPB_SCASE
    default: return nullptr;
    }
}

}  // namespace

size_t small_call_smem_bytes(int n, int w, int threads) { return SmallLayout(n, w, threads).bytes(); }

// Whether the fused call can run on device `dev` (the current one, with
// `sms` SMs) with `blocks` CTAs of `threads` threads all resident at once
// (one CTA per SM); configures the kernel's shared memory on first use.
// Asked once per device, size and shape.
static int small_call_ready(SmallKernel kern, const Problem& pb, int blocks, int threads, int dev, int sms,
                            size_t smem, bool* ok)
{
    *ok = false;
    if (!kern || threads > kSmallCallThreads || threads < 32 || threads % 32 != 0) return SPB_OK;
    if (dev < 0 || dev >= 64 || blocks > sms) return SPB_OK;  // one CTA per SM must hold the whole grid
    static std::mutex mu;
    static int fits[64][kSmallCallMaxN + 1];  // 0 unknown, 1 kernel configured, -1 cannot run
    static signed char resident[64][kSmallCallMaxN + 1][kSmallCallThreads / 32 + 1];  // 0 unknown, 1, -1
    std::lock_guard<std::mutex> lk(mu);
    if (fits[dev][pb.n] == 0) {
        int optin = 0, coop = 0;
        cudaFuncAttributes fa{};
        SPB_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        SPB_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        SPB_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
        fits[dev][pb.n] = -1;
        if (coop) {
            SPB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              optin - (int)fa.sharedSizeBytes));
            fits[dev][pb.n] = 1;
        }
    }
    if (fits[dev][pb.n] < 0) return SPB_OK;
    signed char& res = resident[dev][pb.n][threads / 32];
    if (res == 0) {
        int per_sm = 0;
        SPB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
        res = per_sm >= 1 ? 1 : -1;
    }
    *ok = res > 0;
    return SPB_OK;
}

// Launches the fused call on device `dev` (the current one, with `sms`
// SMs) if it can keep `blocks` CTAs of `threads` threads resident at once;
// *launched tells whether it did.  rb_host (may be null): the device's
// address of a page-locked copy of the readback, which the kernel fills last.
int launch_small_call(const Problem& pb, const double* d_a, const double* a_stage, int blocks, int threads,
                      Readback* rb_host, int dev, int sms, cudaStream_t s, bool* launched)
{
    *launched = false;
    SmallKernel kern = small_kernel(pb.n);
    const size_t smem = small_call_smem_bytes(pb.n, pb.w, threads);
    bool ok = false;
    int st = small_call_ready(kern, pb, blocks, threads, dev, sms, smem, &ok);
    if (st != SPB_OK || !ok) return st;
    Problem p = pb;
    const double* a = d_a;
    const double* as = a_stage;
    Readback* h = rb_host;
    void* args[] = {&p, &a, &as, &h};
    SPB_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(blocks), dim3(threads), args, smem, s));
    *launched = true;
    return SPB_OK;
}

// ---- the call as a CUDA graph --------------------------------------------
// A call issues the events around it and the cooperative launch: several
// microseconds of host time, during which the device waits for the launch.
// Replayed as one graph (the kernel between two events) it costs one graph
// launch.  A
// graph is built for a launch (the kernel's Problem, its matrix, staging and
// readback addresses, the shape) the second time that launch is asked for,
// and kept in a small per-context cache; a matrix given on the device is
// part of the launch, so a caller that passes a new device pointer each time
// keeps the direct path.
namespace {

struct SmallGraph {
    bool valid = false;         // the key below is set
    bool failed = false;        // building the graph failed: use the direct path
    int uses = 0;
    unsigned long long stamp = 0;
    Problem pb{};
    const double* a = nullptr;      // the matrix the kernel reads (or fills from the staging)
    const double* stage = nullptr;  // device address of the page-locked staging (host input) or null
    Readback* rb_host = nullptr;
    int blocks = 0, threads = 0;
    bool timed = true;  // the graph records the context's events around the kernel
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

struct SmallGraphCache {
    SmallGraph e[8];
    unsigned long long clock = 0;
};

void drop(SmallGraph& g)
{
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g = SmallGraph{};
}

void release_cache(void* p)
{
    SmallGraphCache* c = static_cast<SmallGraphCache*>(p);
    if (!c) return;
    for (SmallGraph& g : c->e) drop(g);
    delete c;
}

bool same_launch(const SmallGraph& g, const Problem& pb, const double* a, const double* stage, Readback* rb_host,
                 int blocks, int threads, bool timed)
{
    return g.valid && std::memcmp(&g.pb, &pb, sizeof(Problem)) == 0 && g.a == a && g.stage == stage &&
           g.rb_host == rb_host && g.blocks == blocks && g.threads == threads && g.timed == timed;
}

// Captures events and kernel on the context's own stream.  Any error ends
// the capture and leaves the entry marked failed.
void build(DeviceContext* ctx, SmallGraph& g, SmallKernel kern, size_t smem)
{
    cudaStream_t cs = ctx->stream;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        g.failed = true;
        return;
    }
    Problem p = g.pb;
    const double* a = g.a;
    const double* as = g.stage;
    Readback* h = g.rb_host;
    void* args[] = {&p, &a, &as, &h};
    cudaError_t e = cudaSuccess;
    if (g.timed) e = cudaEventRecordWithFlags(ctx->ev_begin, cs, cudaEventRecordExternal);
    if (e == cudaSuccess)
        e = cudaLaunchCooperativeKernel((const void*)kern, dim3(g.blocks), dim3(g.threads), args, smem, cs);
    if (e == cudaSuccess && g.timed) e = cudaEventRecordWithFlags(ctx->ev_end, cs, cudaEventRecordExternal);
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g.exec, graph, 0);
    g.graph = graph;
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
        g.exec = nullptr;
        g.graph = nullptr;
        g.failed = true;
    }
}

}  // namespace

// The fused call through a cached graph, on stream s.  The kernel reads its
// matrix at d_a; with host input, a_stage (the device address of the
// page-locked staging that holds it) is copied there by the kernel first.
// When timed, the graph also records the context's events ev_begin and
// ev_end around the kernel, which is then the whole call on the device (the
// matrix copy is its first step).  *launched tells whether it ran; when it
// did not, nothing was enqueued.
int launch_small_call_graph(DeviceContext* ctx, const Problem& pb, const double* d_a, const double* a_stage,
                            int blocks, int threads, Readback* rb_host, bool timed, cudaStream_t s,
                            bool* launched)
{
    *launched = false;
    SmallKernel kern = small_kernel(pb.n);
    const size_t smem = small_call_smem_bytes(pb.n, pb.w, threads);
    bool ok = false;
    int st = small_call_ready(kern, pb, blocks, threads, ctx->device, ctx->sm_count, smem, &ok);
    if (st != SPB_OK || !ok) return st;
    if (!ctx->small_graphs) {
        ctx->small_graphs = new SmallGraphCache();
        ctx->release_small_graphs = release_cache;
    }
    SmallGraphCache* c = static_cast<SmallGraphCache*>(ctx->small_graphs);
    SmallGraph* g = nullptr;
    for (SmallGraph& x : c->e)
        if (same_launch(x, pb, d_a, a_stage, rb_host, blocks, threads, timed)) g = &x;
    if (!g) {  // first sight of this launch: remember it, run it directly
        SmallGraph* lru = &c->e[0];
        for (SmallGraph& x : c->e)
            if (!x.valid || x.stamp < lru->stamp) lru = &x;
        if (lru->valid) drop(*lru);
        lru->valid = true;
        lru->pb = pb;
        lru->a = d_a;
        lru->stage = a_stage;
        lru->timed = timed;
        lru->rb_host = rb_host;
        lru->blocks = blocks;
        lru->threads = threads;
        lru->uses = 1;
        lru->stamp = ++c->clock;
        return SPB_OK;
    }
    g->stamp = ++c->clock;
    ++g->uses;
    if (g->failed) return SPB_OK;
    if (!g->exec) {
        build(ctx, *g, kern, smem);
        if (!g->exec) return SPB_OK;
    }
    SPB_CUDA_TRY(cudaGraphLaunch(g->exec, s));
    *launched = true;
    return SPB_OK;
}

}  // namespace dense
}  // namespace spb
