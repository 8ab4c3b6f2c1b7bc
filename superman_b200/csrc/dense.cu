// Dense real and complex permanents: Nijenhuis–Wilf Ryser with Gray-code
// enumeration, restructured for sm_100a.
//
// Reference behaviour (paths relative to the SUPerman tree):
//   x_i = a_{i,n-1} - rowsum_i / 2,   perm = (4(n%2)-2) * sum_S (-1)^|S| prod_i x_i(S)
//   over the subsets S of columns 0..n-2, walked in Gray order
//   (Algorithms/CPU/Dense/dpNaivePerman.h:53-141,
//    Algorithms/GPU/Dense/DenseKernelDefinitions.cuh:189-264).
//
// B200 formulation.  The n-1 column bits of a subset index are split into
//   low  w bits : enumerated from a shared-memory table DE[d][r] holding the
//                 correctly rounded subset sums of the w lowest columns;
//   high bits   : a "unit" index walked in Gray order per thread, with the
//                 unit base vector xtop kept in double-double (hi in registers,
//                 lo in shared memory).
// Every term is x_r = fl(xtop_r + DE[d][r]) — one rounding from exact
// values, so the row sums never drift (the reference accumulates x over
// whole chunks, dpNaivePerman.h:125-129).  All lanes of a warp walk the same
// d at the same time, so DE reads are shared-memory broadcasts.  Terms are
// evaluated in groups of G consecutive d with compile-time signs; each unit's
// FP64 sum is added to a per-thread double-double total, then reduced
// warp -> block -> grid in a fixed order (deterministic).
//
// Rows are pre-scaled by exact powers of two (max |a_rj| in [0.5, 1)) and the
// exponent sum is applied to the final result.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "context.h"
#include "dense_host.h"
#include "dense_impl.cuh"
#include "sparse_impl.cuh"
#include "spb_common.cuh"

namespace spb {
namespace dense {

// ------------------------------------------------------------ setup kernel --
// Builds every table the walk kernels read, one CTA per row r (every value
// below depends on its own row only, apart from the exponent sum, which
// CTA 0 adds up).  Row r is staged in shared memory (CTA 0 stages the whole
// matrix, n*n*comps doubles, for the exponents of every row).
// Per part, one warp builds the row's subset sums DE[d][r] level by level
// behind warp barriers (in shared memory with smem_tables, else in place in
// the global table), another forms the NW start value, and the CTA then
// writes the tables out, the row's bound and its high columns.
//   4 warps: 0, 1 tables (part 0, 1), 2 start values, 3 high columns.
__global__ void __launch_bounds__(128) setup_kernel(Problem pb, const double* __restrict__ a_in, int smem_tables)
{
    const int n = pb.n, c = pb.comps, w = pb.w, G = pb.g;
    const int tid = threadIdx.x, bd = blockDim.x, lane = tid & 31, wid = tid >> 5, r = blockIdx.x;
    const int terms = 1 << w;
    __shared__ int s_eall[kMaxN];
    // CTA 0 stages the whole matrix (it also adds up every row's exponent),
    // the others their row: row r is s_row[0 .. n*c) either way
    extern __shared__ __align__(16) double s_row[];  // [rows][n][c], scaled after step 1; then [c][terms] hi, lo
    double* th = s_row + ((n * n * c + 1) & ~1);
    double* tl = th + (size_t)c * terms;
    const int nst = r == 0 ? n : 1;

    // 0. What the later kernels of the call accumulate into starts at zero.
    if (r == 0) {
        if (tid < 4) pb.ticket[tid] = 0u;
        if (pb.f32 && tid == 0) pb.rb->err = 0.0;  // the FP32 walk's sum of squared terms
        if (pb.mode != 0) {
            for (int i = tid; i < kHistBins; i += bd) {
                pb.hist_s2[i] = 0.0;
                pb.hist_cnt[i] = 0ull;
                pb.pre_cnt[i] = 0u;
            }
            if (tid == 0) {
                *pb.raw_n = 0ull;
                *pb.list_bin = pb.list_bin_init;
            }
        }
    }
    for (int i = tid; i < nst * n * c; i += bd) s_row[i] = a_in[(size_t)r * n * c + i];
    __syncthreads();
    // 1. Row exponents: scale row q by 2^-e_q so that its largest |a_qj| lies
    //    in [0.5, 1); a warp per staged row (fmax does not depend on the
    //    order).  CTA 0 writes their sum.
    for (int q = wid; q < nst; q += bd >> 5) {
        double mx = 0.0;
        for (int j = lane; j < n * c; j += 32) mx = fmax(mx, fabs(s_row[q * n * c + j]));
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        if (lane == 0) {
            int e = 0;
            if (mx > 0.0 && isfinite(mx)) frexp(mx, &e);
            s_eall[q] = e;
        }
    }
    __syncthreads();
    if (r == 0 && wid == 0) {
        int es = 0;
        for (int q = lane; q < n; q += 32) es += s_eall[q];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) es += __shfl_xor_sync(0xffffffffu, es, off);
        if (lane == 0) *pb.exp_sum = es;
    }
    const int er = s_eall[0];
    for (int i = tid; i < n * c; i += bd) {
        const double v = ldexp(s_row[i], -er);
        s_row[i] = v;
        pb.as[(size_t)r * n * c + i] = v;
    }
    __syncthreads();
    // entry d of row r, part p, in the global table [c][terms/G][n][G]
    auto gpos = [&](int p, int d) {
        return (size_t)p * terms * n + (size_t)(d / G) * n * G + (size_t)r * G + (d % G);
    };
    if (wid < c) {
        // 3. Low-column subset sums of part p = wid: the double-double sum
        //    of the selected columns added in ascending order, level by
        //    level: with k the highest bit of d, DE[d] = DE[d - 2^k] + a_k.
        const int p = wid;
        double* hh = th + (size_t)p * terms;
        double* ll = tl + (size_t)p * terms;
        if (smem_tables) {
            if (lane == 0) {
                hh[0] = 0.0;
                ll[0] = 0.0;
            }
            for (int k = 0; k < w; ++k) {
                __syncwarp();  // level k reads the entries of levels < k
                const int half = 1 << k;
                const double ak = s_row[k * c + p];
                for (int e = lane; e < half; e += 32) {
                    const dd v = dd_add_d(dd{hh[e], ll[e]}, ak);
                    hh[half + e] = v.hi;
                    ll[half + e] = v.lo;
                }
            }
        } else {
            if (lane == 0) {
                pb.de_hi[gpos(p, 0)] = 0.0;
                pb.de_lo[gpos(p, 0)] = 0.0;
            }
            for (int k = 0; k < w; ++k) {
                __syncwarp();
                const int half = 1 << k;
                const double ak = s_row[k * c + p];
                for (int e = lane; e < half; e += 32) {
                    const size_t f = gpos(p, e), t = gpos(p, half + e);
                    const dd v = dd_add_d(dd{pb.de_hi[f], pb.de_lo[f]}, ak);
                    pb.de_hi[t] = v.hi;
                    pb.de_lo[t] = v.lo;
                }
            }
        }
    } else if (wid == 2) {
        // 2. NW start value in double-double: x0 = a'_{r,n-1} - rowsum'_r / 2.
        if (lane < c) {
            const int p = lane;
            dd sm = {0.0, 0.0};
            for (int j = 0; j < n; ++j) sm = dd_add_d(sm, s_row[j * c + p]);
            dd h = {-0.5 * sm.hi, -0.5 * sm.lo};  // exact halving
            dd x = dd_add_d(h, s_row[(n - 1) * c + p]);
            pb.x0_hi[p * n + r] = x.hi;
            pb.x0_lo[p * n + r] = x.lo;
        }
    } else if (wid == 3) {
        // 4. High columns, column-major: mt[part][j][r] = a'_{r, w+j}.
        const int ntop = n - 1 - w;
        for (int i = lane; i < ntop * c; i += 32) {
            const int p = i / ntop, j = i % ntop;
            pb.mt[((size_t)p * ntop + j) * n + r] = s_row[(w + j) * c + p];
        }
        // real row bound [sum_j min(0,a'_rj), sum_j max(0,a'_rj)] over the low columns
        if (c == 1 && lane == 0) {
            double lo = 0.0, hi = 0.0;
            for (int j = 0; j < w; ++j) {
                const double v = s_row[j];
                if (v < 0.0) lo += v; else hi += v;
            }
            pb.bnd[r] = lo;
            pb.bnd[n + r] = hi;
        }
    }
    __syncthreads();
    // write-out of the tables (the row's entries sit in runs of G), and the
    // FP32 copy of the hi words for the FP32-product walk
    if (smem_tables)
        for (int i = tid; i < c * terms; i += bd) {
            const int p = i / terms, d = i % terms;
            const size_t t = gpos(p, d);
            pb.de_hi[t] = th[i];
            pb.de_lo[t] = tl[i];
        }
    if (pb.de32)
        for (int i = tid; i < c * terms; i += bd) {
            const int p = i / terms, d = i % terms;
            const size_t t = gpos(p, d);
            pb.de32[t] = __double2float_rn(smem_tables ? th[i] : pb.de_hi[t]);
        }
    // complex row bound: max_d |DE[d][r]|, a warp's maximum over d (the bit
    // patterns of non-negative doubles order like the values)
    if (c == 2 && wid == 0) {
        unsigned long long mx = 0ull;
        for (int d = lane; d < terms; d += 32) {
            const double re = smem_tables ? th[d] : pb.de_hi[gpos(0, d)];
            const double im = smem_tables ? th[terms + d] : pb.de_hi[gpos(1, d)];
            mx = max(mx, (unsigned long long)__double_as_longlong(hypot(re, im)));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0) pb.bnd[r] = __longlong_as_double((long long)mx) * (1.0 + 0x1p-50);
    }
}

}  // namespace dense
}  // namespace spb

// ======================================================================
// Host drivers
// ======================================================================
namespace spb {
namespace dense {

// The staged matrix (CTA 0 stages all of it), rounded up to an even count of
// doubles (a row's tables follow it on a 16-byte boundary).
size_t setup_smem_bytes(int n, int comps) { return sizeof(double) * (((size_t)n * n * comps + 1) & ~(size_t)1); }

// The fused small-matrix call (small_call.cu).
constexpr int kSmallCallMaxN = 26;
size_t small_call_smem_bytes(int n, int w, int threads);
int launch_small_call(const Problem& pb, const double* d_a, const double* a_stage, int blocks, int threads,
                      Readback* rb_host, int dev, int sms, cudaStream_t s, bool* launched);
int launch_small_call_graph(DeviceContext* ctx, const Problem& pb, const double* d_a, const double* a_stage,
                            int blocks, int threads, Readback* rb_host, bool timed, cudaStream_t s,
                            bool* launched);

// The staged matrix plus, when they fit, one row's subset-sum tables: the setup
// kernel's dynamic shared-memory limit is raised to the maximum once per
// device (which also loads the kernel); *limit receives it.
int prepare_setup(int* limit)
{
    static std::mutex mu;
    static int room[64] = {0};
    int dev = 0;
    SPB_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (room[dev & 63] == 0) {
        int optin = 0;
        cudaFuncAttributes fa{};
        SPB_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        SPB_CUDA_TRY(cudaFuncGetAttributes(&fa, setup_kernel));
        SPB_CUDA_TRY(cudaFuncSetAttribute(setup_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          optin - (int)fa.sharedSizeBytes));
        room[dev & 63] = optin - (int)fa.sharedSizeBytes;
    }
    if (limit) *limit = room[dev & 63];
    return SPB_OK;
}

int launch_setup(const Problem& pb, const double* d_a, cudaStream_t s)
{
    int limit = 0;
    int st = prepare_setup(&limit);
    if (st != SPB_OK) return st;
    const size_t base = setup_smem_bytes(pb.n, pb.comps);
    const size_t tables = sizeof(double) * 2 * (size_t)pb.comps * ((size_t)1 << pb.w);  // one row's
    const int smem_tables = base + tables <= (size_t)limit ? 1 : 0;
    setup_kernel<<<pb.n, 128, base + (smem_tables ? tables : 0), s>>>(pb, d_a, smem_tables);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

// Terms per group in the walk kernels; must equal RealCfg<N>::G /
// ComplexCfg<N>::G, and the unit (2^w terms) must hold at least one group.
int group_size(int n, int comps)
{
    if (comps == 1) return n >= 3 ? 4 : (n == 2 ? 2 : 1);
    return ComplexGroup(n);
}

int choose_unit_bits(int n, int comps, const spb_options* opt)
{
    int w;
    if (opt && opt->unit_bits > 0) {
        w = opt->unit_bits;
    } else {
        // Table budget 64 KB per part; keep >= 2^16 units when n allows.
        w = 8;
        while (w > 2 && ((size_t)1 << w) * n * 8 * comps > (size_t)64 * 1024) --w;
        while (w > 2 && (n - 1 - w) < 16 && w > (n - 1) - 16) --w;
    }
    if (w > n - 1) w = n - 1;
    const int g = group_size(n, comps);
    const int wmin = g == 4 ? 2 : (g == 2 ? 1 : 0);
    if (w < wmin) w = wmin;
    return w;
}

// Sizes the scratch arena and fills the device pointers of *pb.
size_t plan_layout(Problem* pb, char* base, size_t* in_offset)
{
    const int n = pb->n, c = pb->comps;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    size_t o_in = take(sizeof(double) * n * n * c);
    size_t o_as = take(sizeof(double) * n * n * c);
    size_t o_x0h = take(sizeof(double) * n * c);
    size_t o_x0l = take(sizeof(double) * n * c);
    size_t terms = (size_t)1 << pb->w;
    size_t o_deh = take(sizeof(double) * terms * n * c);
    size_t o_del = take(sizeof(double) * terms * n * c);
    const bool f32 = pb->f32 != 0;
    size_t o_d32 = f32 ? take(sizeof(float) * terms * n * c) : 0;
    size_t o_mt = take(sizeof(double) * (size_t)(n - 1 - pb->w > 0 ? n - 1 - pb->w : 1) * n * c);
    // two per CTA at least: the fused small call keeps its walk totals and its
    // corrections apart
    size_t o_part = take(sizeof(dd) * (size_t)pb->grid * (c > 2 ? c : 2));
    size_t o_tick = take(sizeof(unsigned) * 4);
    size_t o_rbk = take(sizeof(Readback));
    size_t o_bnd = take(sizeof(double) * 2 * n);
    size_t o_hs = take(sizeof(double) * kHistBins);
    size_t o_hc = take(sizeof(unsigned long long) * kHistBins);
    const size_t T = (size_t)pb->grid * pb->threads;
    const bool refine = pb->mode != 0;
    size_t o_tm = refine ? take(sizeof(unsigned short) * T) : 0;
    size_t o_pc = refine ? take(sizeof(unsigned) * kHistBins) : 0;
    size_t o_lb = refine ? take(sizeof(int) * 4) : 0;
    size_t o_rn = refine ? take(sizeof(unsigned long long) * 2) : 0;
    size_t o_ru = refine ? take(sizeof(unsigned long long) * kRawCap) : 0;
    size_t o_rb = refine ? take(sizeof(unsigned short) * kRawCap) : 0;
    if (base) {
        pb->tmax = refine ? reinterpret_cast<unsigned short*>(base + o_tm) : nullptr;
        pb->pre_cnt = refine ? reinterpret_cast<unsigned*>(base + o_pc) : nullptr;
        pb->list_bin = refine ? reinterpret_cast<int*>(base + o_lb) : nullptr;
        pb->raw_n = refine ? reinterpret_cast<unsigned long long*>(base + o_rn) : nullptr;
        pb->raw_cap = refine ? kRawCap : 0;
        pb->raw_u = refine ? reinterpret_cast<unsigned long long*>(base + o_ru) : nullptr;
        pb->raw_b = refine ? reinterpret_cast<unsigned short*>(base + o_rb) : nullptr;
        pb->bnd = reinterpret_cast<double*>(base + o_bnd);
        pb->hist_s2 = reinterpret_cast<double*>(base + o_hs);
        pb->hist_cnt = reinterpret_cast<unsigned long long*>(base + o_hc);
        pb->as = reinterpret_cast<double*>(base + o_as);
        pb->x0_hi = reinterpret_cast<double*>(base + o_x0h);
        pb->x0_lo = reinterpret_cast<double*>(base + o_x0l);
        pb->de_hi = reinterpret_cast<double*>(base + o_deh);
        pb->de_lo = reinterpret_cast<double*>(base + o_del);
        pb->de32 = f32 ? reinterpret_cast<float*>(base + o_d32) : nullptr;
        pb->mt = reinterpret_cast<double*>(base + o_mt);
        pb->partials = reinterpret_cast<dd*>(base + o_part);
        pb->ticket = reinterpret_cast<unsigned*>(base + o_tick);
        pb->rb = reinterpret_cast<Readback*>(base + o_rbk);
        pb->result = pb->rb->res;
        pb->exp_sum = &pb->rb->exp_sum;
        pb->list_n = &pb->rb->list_n;
    }
    if (in_offset) *in_offset = o_in;
    return off;
}

size_t walk_smem_bytes(const Problem& pb, int threads)
{
    const int n = pb.n, c = pb.comps;
    if (pb.na < n) return sparse_smem_bytes(n, pb.na, pb.w, threads);
    size_t terms = (size_t)1 << pb.w;
    int ntop = n - 1 - pb.w;
    return sizeof(double) * (terms * n * c + (size_t)(ntop > 0 ? ntop : 0) * n * c +
                             (size_t)n * c * threads) +
           kHistSmemBytes + bound_smem_bytes(n);
}

int run(const double* a, bool a_on_device, int n, int comps, const spb_options* opt_in, spb_result* out,
        const WalkPlan* plan, DeviceContext* own_ctx)
{
    double t_start = wall_seconds();
    if (!out) {
        spb_set_error("null result pointer");
        return SPB_ERR_INVALID;
    }
    std::memset(out, 0, sizeof(*out));
    spb_options opt;
    if (opt_in) opt = *opt_in; else spb_default_options(&opt);
    if (!a || n < 1 || n > kMaxN) {
        spb_set_error("dense permanent needs a non-null matrix and 1 <= n <= %d (got n=%d)", kMaxN, n);
        return out->status = SPB_ERR_INVALID;
    }
    int st = SPB_OK;
    DeviceContext* ctx = own_ctx ? own_ctx : get_context(opt.device, &st);
    if (!ctx) return out->status = st;
    std::lock_guard<std::mutex> lk(ctx->mu);
    SPB_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t stream = call_stream(ctx, &opt);

    Problem pb{};
    pb.n = n;
    pb.na = n;
    pb.comps = comps;
    pb.w = choose_unit_bits(n, comps, &opt);
    if (opt.precision == SPB_PREC_FP32) {
        if (n > kMaxF32N || n < 3) {
            spb_set_error("FP32 products are offered for 3 <= n <= %d (got n=%d)", kMaxF32N, n);
            return out->status = SPB_ERR_INVALID;
        }
        pb.f32 = 1;
        plan = nullptr;  // the FP32 variant is the dense walk
    }
    if (plan && plan->na < n) {
        if (comps != 1 || plan->na < 1 || plan->na > kMaxActive || plan->w < 2 || plan->w > n - 2) {
            spb_set_error("row-compacted walk: bad plan (n=%d, active rows %d, w=%d)", n, plan->na, plan->w);
            return out->status = SPB_ERR_INVALID;
        }
        pb.na = plan->na;
        pb.w = plan->w;
    }
    pb.g = group_size(n, comps);
    pb.units = 1ull << (n - 1 - pb.w);

    auto smem_for = [&](int th) { return pb.f32 ? walk_f32_smem_bytes(pb, th) : walk_smem_bytes(pb, th); };
    int threads = opt.threads_per_block > 0 ? opt.threads_per_block : 0;
    const int max_threads = pb.f32 ? walk_f32_max_threads(n, comps) : (pb.na < n ? 512 : walk_max_threads(n, comps));
    if (threads == 0) {
        threads = max_threads;
        // fit the per-thread lo vectors next to the tables
        while (threads > 64 && smem_for(threads) > ctx->smem_optin) threads -= 32;
    }
    if (threads > max_threads) threads = max_threads;
    threads = (threads / 32) * 32;
    if (threads < 32) threads = 32;
    size_t smem = smem_for(threads);
    if (smem > ctx->smem_optin) {
        spb_set_error("dense n=%d: %zu B shared memory exceeds the %zu B limit", n, smem, ctx->smem_optin);
        return out->status = SPB_ERR_INVALID;
    }
    // The fused small call (below) walks with fewer threads per CTA on every
    // SM when the units would leave SMs idle at full CTAs (n = 19 .. 25:
    // 2^15 or 2^16 units fill 64 or 128 CTAs of 512 threads; 147 CTAs of 448
    // threads give each SM an eighth less to walk).
    const bool small_candidate = opt.small_call >= 0 && comps == 1 && pb.na == n && !pb.f32 && n >= 4 &&
                                 n <= kSmallCallMaxN && !opt.replay_listing;
    if (small_candidate && opt.threads_per_block <= 0 && opt.blocks <= 0) {
        if (pb.units >= 256ull * (unsigned long long)ctx->sm_count) {
            const unsigned long long per_sm = (pb.units + ctx->sm_count - 1) / ctx->sm_count;
            const int t = (int)((per_sm + 31) / 32 * 32);
            if (t <= threads) threads = t;
        }
        // the fused kernel's tables, warp bases and histogram fit one CTA
        // (n = 26: 480 threads; its 2^17 units then take two passes)
        while (threads > 256 && small_call_smem_bytes(n, pb.w, threads) > ctx->smem_optin) threads -= 32;
        smem = smem_for(threads);
    }
    int blocks = opt.blocks > 0 ? opt.blocks : ctx->sm_count;
    // never launch more threads than units
    unsigned long long max_blocks = (pb.units + threads - 1) / threads;
    if ((unsigned long long)blocks > max_blocks) blocks = (int)max_blocks;
    if (blocks < 1) blocks = 1;
    pb.grid = blocks;
    pb.threads = threads;
    const bool dd_mode = opt.precision == SPB_PREC_DD;
    pb.mode = dd_mode ? 1 : 0;
    if (dd_mode && pb.na == n) {
        // the refinement stages both table words of every part (256 threads
        // at the least): refuse before any launch when they cannot fit
        const size_t rs = refine_smem_bytes(pb, 256);
        if (rs + 2048 > ctx->smem_optin) {
            spb_set_error("dense n=%d, unit_bits=%d: the double-double refinement needs %zu B shared memory "
                          "(limit %zu B); use fewer unit bits", n, pb.w, rs, ctx->smem_optin);
            return out->status = SPB_ERR_INVALID;
        }
    }

    size_t in_off = 0;
    size_t need = plan_layout(&pb, nullptr, &in_off);
    if ((st = ensure_scratch(ctx, need)) != SPB_OK) return out->status = st;
    char* base = static_cast<char*>(ctx->scratch);
    plan_layout(&pb, base, &in_off);
    // page-locked: the readback, then (fused small call) a staging copy of a
    // host matrix
    constexpr size_t kStageOff = 256;
    static_assert(sizeof(Readback) <= kStageOff, "readback fits before the staging area");
    const size_t a_bytes = sizeof(double) * n * n * comps;
    if ((st = ensure_pinned(ctx, kStageOff + a_bytes)) != SPB_OK) return out->status = st;
    Readback* hrb = static_cast<Readback*>(ctx->pinned);
    // The refinement list is sized before the walk for the threshold's cap
    // (1/8 of the units), up to 2^21 units; a larger count is met after the
    // readback with a larger list.
    const size_t entry = sizeof(double) * 2 * n * comps;
    if (dd_mode) {
        const unsigned long long cap = std::min<unsigned long long>(pb.units / 8 + 1, 1ull << 21);
        if ((st = ensure_list(ctx, cap * sizeof(unsigned long long) + 256)) != SPB_OK) return out->status = st;
        pb.list_u = static_cast<unsigned long long*>(ctx->list);
        pb.list_cap = cap;
        pb.list_x = nullptr;
        pb.tol = opt.rel_tol > 0.0 ? opt.rel_tol : 1e-13;
    }
    double* d_in = reinterpret_cast<double*>(base + in_off);
    const double* d_a = a_on_device ? a : d_in;
    dd res[2] = {{0.0, 0.0}, {0.0, 0.0}};
    int exp_sum = 0, launches = 0;
    double ms_refine = 0.0;
    // Small real matrices: the whole call as one cooperative kernel
    // (small_call.cu), unless the device cannot hold its grid or its count
    // check fails, in which case the separate kernels below run.  The kernel
    // writes the finished readback straight into the pinned buffer when the
    // device can address it (no copy after the kernel), and takes a host
    // matrix from the pinned staging area itself (no copy before it: a copy
    // engine takes several microseconds to start for 4.6 KB).  A launch asked
    // for again is replayed as a CUDA graph (events and kernel; the kernel
    // alone with skip_timing).
    const bool fused_fits = small_candidate && pb.units <= kRawCap &&
                            small_call_smem_bytes(n, pb.w, threads) <= ctx->smem_optin;
    Readback* mapped = static_cast<Readback*>(ctx->pinned_dev);
    const double* a_stage = nullptr;  // device address of the staged host matrix
    if (fused_fits && mapped && !a_on_device) {
        std::memcpy(static_cast<char*>(ctx->pinned) + kStageOff, a, a_bytes);
        a_stage = reinterpret_cast<const double*>(static_cast<char*>(ctx->pinned_dev) + kStageOff);
    }
    bool fused = false, graphed = false;
    if (fused_fits && mapped) {
        if ((st = launch_small_call_graph(ctx, pb, d_a, a_stage, blocks, threads, mapped, !opt.skip_timing, stream,
                                          &fused)) != SPB_OK)
            return out->status = st;
        graphed = fused;
    }
    if (!graphed) {
        SPB_CUDA_TRY(cudaEventRecord(ctx->ev_call0, stream));
        if (!a_on_device && !a_stage)
            SPB_CUDA_TRY(cudaMemcpyAsync(d_in, a, a_bytes, cudaMemcpyHostToDevice, stream));
        if (fused_fits) {
            SPB_CUDA_TRY(cudaEventRecord(ctx->ev_begin, stream));
            if ((st = launch_small_call(pb, d_a, a_stage, blocks, threads, mapped, ctx->device, ctx->sm_count,
                                        stream, &fused)) != SPB_OK)
                return out->status = st;
            if (fused) {
                SPB_CUDA_TRY(cudaEventRecord(ctx->ev_end, stream));
                SPB_CUDA_TRY(cudaEventRecord(ctx->ev_call1, stream));
            }
        }
        // the fused call did not run: the separate kernels read the matrix at d_in
        if (!fused && a_stage) SPB_CUDA_TRY(cudaMemcpyAsync(d_in, a, a_bytes, cudaMemcpyHostToDevice, stream));
    }
    if (fused) {
        if (!mapped) SPB_CUDA_TRY(cudaMemcpyAsync(hrb, pb.rb, sizeof(Readback), cudaMemcpyDeviceToHost, stream));
        SPB_CUDA_TRY(cudaStreamSynchronize(stream));
        launches = 1;
        res[0] = dd_add(hrb->res[0], hrb->corr[0]);
        exp_sum = hrb->exp_sum;
        if (dd_mode) {
            out->err_est = hrb->err;
            out->refined_units = hrb->count;
            if (hrb->list_n != hrb->count) fused = false;  // run the separate kernels instead
        }
    }
    if (!fused) {
    // after a replayed fused call whose count check failed, the call's device
    // span is timed from here (the graph records no ev_call0)
    if (graphed) SPB_CUDA_TRY(cudaEventRecord(ctx->ev_call0, stream));
    // The walk's list bin, written by the setup kernel (which also zeroes the
    // counters and histograms): 0 lists every unit when all fit the list;
    // 0x7f7f7f7f, above every bin, lists none (the row-compacted walk, whose
    // refinement goes through the scan); with a bound pass pick_list_bin
    // overwrites it.
    pb.list_bin_init = (pb.na == n && pb.units <= pb.raw_cap / 2) ? 0 : 0x7f7f7f7f;
    if ((st = launch_setup(pb, d_a, stream)) != SPB_OK) return out->status = st;
    SPB_CUDA_TRY(cudaGetLastError());
    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_begin, stream));
    launches = 2;
    if (dd_mode && pb.na == n && pb.units > pb.raw_cap / 2) {
        // Size the first pass's unit list from a bound-only pass (about 1.5 %
        // of a dense walk).  The row-compacted walk has few terms per unit, so
        // there the pass would cost a large share; it lists nothing and a
        // refinement, when one is needed, goes through the scan.
        if ((st = launch_bound_pass(pb, blocks, stream)) != SPB_OK) return out->status = st;
        launches += 2;
    }
    st = pb.f32 ? launch_walk_f32(pb, blocks, threads, smem, stream) : launch_walk(pb, blocks, threads, smem, stream);
    if (st != SPB_OK) return out->status = st;
    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_end, stream));

    // Double-double: threshold, listing and refinement follow the walk on the
    // stream; the host reads everything back once.
    auto enqueue_refinement = [&]() -> int {
        int r;
        if ((r = launch_listing(pb, stream)) != SPB_OK) return r;
        if ((r = launch_refine(pb, blocks, stream)) != SPB_OK) return r;
        SPB_CUDA_TRY(cudaEventRecord(ctx->ev_ref1, stream));
        launches += 2;
        return SPB_OK;
    };
    auto read_back = [&]() -> int {
        SPB_CUDA_TRY(cudaEventRecord(ctx->ev_call1, stream));
        SPB_CUDA_TRY(cudaMemcpyAsync(hrb, pb.rb, sizeof(Readback), cudaMemcpyDeviceToHost, stream));
        SPB_CUDA_TRY(cudaStreamSynchronize(stream));
        return SPB_OK;
    };
    bool refined = false;
    if (dd_mode) {
        SPB_CUDA_TRY(cudaEventRecord(ctx->ev_ref0, stream));
        if ((st = launch_threshold(pb, stream)) != SPB_OK) return out->status = st;
        launches += 1;
        if (!opt.replay_listing) {
            if ((st = enqueue_refinement()) != SPB_OK) return out->status = st;
            refined = true;
        }
    }
    if ((st = read_back()) != SPB_OK) return out->status = st;
    const dd res0[2] = {hrb->res[0], hrb->res[1]};
    res[0] = res0[0];
    res[1] = res0[1];
    exp_sum = hrb->exp_sum;
    if (dd_mode) {
        const unsigned long long count = hrb->count;
        out->err_est = hrb->err;
        bool ok = refined && hrb->list_n == count && count <= pb.list_cap;
        if (!ok && refined && count > pb.list_cap) {
            // more units than the list was sized for: the same listing, larger list
            if ((st = ensure_list(ctx, count * sizeof(unsigned long long) + 256)) != SPB_OK)
                return out->status = st;
            pb.list_u = static_cast<unsigned long long*>(ctx->list);
            pb.list_cap = count;
            SPB_CUDA_TRY(cudaEventRecord(ctx->ev_ref0, stream));
            SPB_CUDA_TRY(cudaMemsetAsync(pb.list_n, 0, sizeof(unsigned long long), stream));
            if ((st = enqueue_refinement()) != SPB_OK) return out->status = st;
            if ((st = read_back()) != SPB_OK) return out->status = st;
            ok = hrb->list_n == count;
        }
        if (!ok) {
            // Replay the walk (mode 2, same launch shape, so the unit bases
            // are the walk's own) and list the units with their bases.
            if ((st = ensure_list(ctx, count * (entry + sizeof(unsigned long long)) + 256)) != SPB_OK)
                return out->status = st;
            pb.mode = 2;
            pb.thr_bin = hrb->thr;
            pb.list_cap = count;
            pb.list_u = static_cast<unsigned long long*>(ctx->list);
            pb.list_x = reinterpret_cast<double*>(static_cast<char*>(ctx->list) +
                                                  align_up(count * sizeof(unsigned long long), 256));
            SPB_CUDA_TRY(cudaEventRecord(ctx->ev_ref0, stream));
            SPB_CUDA_TRY(cudaMemsetAsync(pb.list_n, 0, sizeof(unsigned long long), stream));
            if (count > 0 && (st = launch_walk(pb, blocks, threads, smem, stream)) != SPB_OK)
                return out->status = st;
            if ((st = launch_refine(pb, blocks, stream)) != SPB_OK) return out->status = st;
            SPB_CUDA_TRY(cudaEventRecord(ctx->ev_ref1, stream));
            launches += count > 0 ? 2 : 1;
            if ((st = read_back()) != SPB_OK) return out->status = st;
            if (hrb->list_n != count) {
                spb_set_error("refinement listed %llu units, histogram counted %llu",
                              (unsigned long long)hrb->list_n, (unsigned long long)count);
                return out->status = SPB_ERR_CUDA;
            }
        }
        for (int cc = 0; cc < comps; ++cc) res[cc] = dd_add(res0[cc], hrb->corr[cc]);
        out->refined_units = count;
        float mr = 0.f;
        if (!opt.skip_timing) SPB_CUDA_TRY(cudaEventElapsedTime(&mr, ctx->ev_ref0, ctx->ev_ref1));
        ms_refine = mr;
    }
    }  // separate kernels
    float ms = 0.f, ms_call = 0.f;
    if (!opt.skip_timing) {
        SPB_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev_begin, ctx->ev_end));
        // a replayed fused call is one kernel, which copies its own input
        if (graphed && fused) ms_call = ms;
        else SPB_CUDA_TRY(cudaEventElapsedTime(&ms_call, ctx->ev_call0, ctx->ev_call1));
    }

    // FP32 products: estimated relative error of the result from the sum of
    // squared terms s2 the walk accumulated.  A term carries k roundings of
    // relative size up to 2^-24 (k = 2n real: n adds and n-1 multiplies; 4n
    // complex), modelled as independent and uniform, so the error of the sum
    // has standard deviation sqrt(s2 * k / 3) * 2^-24.
    int f32_status = SPB_OK;
    if (pb.f32) {
        const double k = (comps == 1 ? 2.0 : 4.0) * n;
        const double mag = comps == 1 ? std::fabs(res[0].hi) : std::hypot(res[0].hi, res[1].hi);
        const double e = std::sqrt(hrb->err * k / 3.0) * 0x1p-24 / mag;
        out->err_est = std::isfinite(e) ? e : HUGE_VAL;
        const double bound = opt.rel_tol > 0.0 ? opt.rel_tol : kF32DefaultBound;
        if (!(out->err_est <= bound)) {
            spb_set_error("FP32 products: estimated relative error %.2e exceeds the bound %.2e (rel_tol); "
                          "the result is returned but not within it: use SPB_PREC_FP64 or SPB_PREC_DD, "
                          "or a looser rel_tol", out->err_est, bound);
            f32_status = SPB_ERR_ACCURACY;
        }
    }

    // perm = (4(n%2)-2) * total * 2^E ; the factor is +-2, an exact power of two.
    const int e = exp_sum + 1;
    const double sgn = (n % 2) ? 1.0 : -1.0;
    out->value = sgn * std::ldexp(res[0].hi, e);
    out->value_lo = sgn * std::ldexp(res[0].lo, e);
    if (comps == 2) {
        out->imag = sgn * std::ldexp(res[1].hi, e);
        out->imag_lo = sgn * std::ldexp(res[1].lo, e);
    }
    out->kernel_s = (ms + ms_refine) * 1e-3;
    out->device_s = ms_call * 1e-3;
    out->gray_steps = (uint64_t)n << (n - 1);
    out->launches = launches;
    out->active_rows = pb.na;
    out->status = f32_status;
    out->elapsed_s = wall_seconds() - t_start;
    return f32_status;
}

}  // namespace dense
}  // namespace spb

extern "C" int spb_perm_dense_f64(const double* a, int n, const spb_options* opt_in, spb_result* out)
{
    spb_options opt;
    if (opt_in) opt = *opt_in; else spb_default_options(&opt);
    return spb::dense::run_real_host(a, n, &opt, out);
}

extern "C" int spb_perm_dense_f64_dev(const double* d_a, int n, const spb_options* opt,
                                      spb_result* out)
{
    return spb::dense::run(d_a, true, n, 1, opt, out, nullptr);
}

extern "C" int spb_perm_dense_c128(const double* a, int n, const spb_options* opt, spb_result* out)
{
    return spb::dense::run(a, false, n, 2, opt, out, nullptr);
}

extern "C" int spb_perm_dense_c128_dev(const double* d_a, int n, const spb_options* opt,
                                       spb_result* out)
{
    return spb::dense::run(d_a, true, n, 2, opt, out, nullptr);
}
