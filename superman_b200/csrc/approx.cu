// Monte-Carlo permanent of a sparse 0/1 pattern: sequential importance
// sampling with per-row scaling and degree-1 propagation.
//
// Reference behaviour (paths relative to the SUPerman tree): aspSingleGPU
// (Algorithms/GPU/Sparse/aspSingleGPU.cuh:45-165) with the kernel
// rasmussenScaleAB (Algorithms/GPU/Sparse/ApproximateSparseKernelDefinitions.cuh:
// 177-290).  The estimate is of the number of perfect matchings of the
// nonzero pattern (the values are not used), one sample at a time:
//   * the pattern is first scaled towards doubly stochastic on the host
//     (INITIAL_BETA = 50 alternating column/row passes, :32-61);
//   * for each row i in order: BETA = 10 passes rescale the columns of row i
//     and then row i itself (:63-122), so the remaining entries of row i,
//     rv_i * cv_j, sum to one; a column is drawn with that probability and
//     the estimate is multiplied by its inverse;
//   * the drawn row and column leave the matrix, and rows or columns left
//     with a single entry are matched at once (:124-172); a line left with
//     none, or a zero scaling sum, makes the sample's estimate 0.
// The mean of the estimates is unbiased.
//
// B200 formulation.  One thread per sample stream; sample k always draws from
// its own SplitMix64 stream seeded by (seed, k), and every floating-point
// operation is an explicitly rounded add, multiply or divide, so a sample's
// estimate does not depend on the launch shape, and the CPU restatement in the
// oracle reproduces it bit for bit.  Per-thread state (scales, remaining
// degrees, the propagation stack) lives in global memory laid out [i][thread],
// so threads that work on the same row touch consecutive words.  Per-thread
// sums of the estimates and of their squares are reduced deterministically.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "context.h"
#include "spb_common.cuh"

namespace spb {
namespace approx {

constexpr int kBeta = 10;         // per-row scaling passes
constexpr int kInitialBeta = 50;  // host scaling passes

struct Pattern {
    int n;
    const int* rptr;  // CSR
    const int* col;
    const int* cptr;  // CSC
    const int* row;
    const float* rv0;  // host-scaled start
    const float* cv0;
};

__host__ __device__ __forceinline__ unsigned long long splitmix_next(unsigned long long& s)
{
    s += 0x9E3779B97F4A7C15ull;
    unsigned long long z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform in (0, 1], 24 bits.
__host__ __device__ __forceinline__ float uniform01(unsigned long long& s)
{
    return (float)((splitmix_next(s) >> 40) + 1ull) * 0x1p-24f;
}

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float frecip(float a) { return __fdiv_rn(1.0f, a); }

// Strided per-thread arrays: element i of thread t at [i * T + t].
struct Lane {
    float* rv;
    float* cv;
    int* re;  // remaining entries per row
    int* ce;  // remaining entries per column
    int* stk;
    unsigned long long T, t;
    __device__ __forceinline__ float& RV(int i) const { return rv[(size_t)i * T + t]; }
    __device__ __forceinline__ float& CV(int j) const { return cv[(size_t)j * T + t]; }
    __device__ __forceinline__ int& RE(int i) const { return re[(size_t)i * T + t]; }
    __device__ __forceinline__ int& CE(int j) const { return ce[(size_t)j * T + t]; }
    __device__ __forceinline__ int& STK(int k) const { return stk[(size_t)k * T + t]; }
};

// Degree-1 propagation after line `start` left (rasmussenScaleAB's d1Reduce,
// :124-172).  `by_col`: start is a column; its rows lose an entry, and a row
// left with one entry is matched to it, which removes that column in turn.
// Otherwise the same with rows and columns exchanged.  Returns true when a
// line is left with no entry (no perfect matching remains).
__device__ bool propagate(const Pattern& P, const Lane& L, int start, bool by_col)
{
    const int* optr = by_col ? P.cptr : P.rptr;  // lines crossing a removed line
    const int* oidx = by_col ? P.row : P.col;
    const int* sptr = by_col ? P.rptr : P.cptr;  // entries of a crossing line
    const int* sidx = by_col ? P.col : P.row;
    int sp = 1;
    L.STK(0) = start;
    for (int ii = 0; ii < sp; ++ii) {
        const int j = L.STK(ii);
        for (int q = optr[j]; q < optr[j + 1]; ++q) {
            const int i = oidx[q];
            float& si = by_col ? L.RV(i) : L.CV(i);
            if (si == 0.0f) continue;
            int& cnt = by_col ? L.RE(i) : L.CE(i);
            const int k = --cnt;
            if (k == 0) return true;
            if (k != 1) continue;
            for (int p = sptr[i]; p < sptr[i + 1]; ++p) {
                const int j2 = sidx[p];
                float& sj = by_col ? L.CV(j2) : L.RV(j2);
                if (sj == 0.0f) continue;
                si = 0.0f;
                sj = 0.0f;
                L.STK(sp++) = j2;
                break;
            }
        }
    }
    return false;
}

// One sample's estimate (0 when the drawn partial matching cannot be
// completed).
__device__ double sample_estimate(const Pattern& P, const Lane& L, unsigned long long seed, unsigned long long k)
{
    const int n = P.n;
    for (int i = 0; i < n; ++i) {
        L.RE(i) = P.rptr[i + 1] - P.rptr[i];
        L.CE(i) = P.cptr[i + 1] - P.cptr[i];
        L.RV(i) = P.rv0[i];
        L.CV(i) = P.cv0[i];
    }
    unsigned long long rng = seed ^ (k * 0xD1B54A32D192ED03ull);
    double est = 1.0;
    for (int i = 0; i < n; ++i) {
        for (int it = 0; it < kBeta; ++it) {
            for (int p = P.rptr[i]; p < P.rptr[i + 1]; ++p) {
                const int j = P.col[p];
                if (L.CV(j) == 0.0f) continue;
                float s = 0.0f;
                for (int q = P.cptr[j]; q < P.cptr[j + 1]; ++q) s = fadd(s, L.RV(P.row[q]));
                if (s == 0.0f) return 0.0;
                L.CV(j) = frecip(s);
            }
            if (L.RV(i) != 0.0f) {
                float s = 0.0f;
                for (int p = P.rptr[i]; p < P.rptr[i + 1]; ++p) s = fadd(s, L.CV(P.col[p]));
                if (s == 0.0f) return 0.0;
                L.RV(i) = frecip(s);
            }
        }
        const float ri = L.RV(i);
        if (ri == 0.0f) continue;  // matched by propagation
        const float u = uniform01(rng);
        float run = 0.0f, prob = 0.0f;
        int chosen = -1;
        for (int p = P.rptr[i]; p < P.rptr[i + 1]; ++p) {
            const int j = P.col[p];
            const float cj = L.CV(j);
            if (cj == 0.0f) continue;
            prob = fmul(ri, cj);
            run = fadd(run, prob);
            chosen = j;
            if (run > u) break;  // else, rounding left the total below u: the last column
        }
        if (chosen < 0) return 0.0;
        est = __dmul_rn(est, __ddiv_rn(1.0, (double)prob));
        L.RV(i) = 0.0f;
        L.CV(chosen) = 0.0f;
        if (propagate(P, L, chosen, true) || propagate(P, L, i, false)) return 0.0;
    }
    return est;
}

struct Sums {
    double* part;            // [grid][2] per-CTA sum and sum of squares
    unsigned* ticket;
    double* total;           // [2]
    double* per_sample;      // optional: estimates of samples [first, first + count)
};

__global__ void __launch_bounds__(128, 8) rasmussen_kernel(Pattern P, Lane L0, unsigned long long first,
                                                        unsigned long long count, unsigned long long seed, Sums S)
{
    Lane L = L0;
    L.T = (unsigned long long)gridDim.x * blockDim.x;
    L.t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    double s1 = 0.0, s2 = 0.0;
    for (unsigned long long k = L.t; k < count; k += L.T) {
        const double e = sample_estimate(P, L, seed, first + k);
        if (S.per_sample) S.per_sample[k] = e;
        s1 += e;
        s2 = __fma_rn(e, e, s2);
    }
    // deterministic reduction: warp shuffles, then CTA, then the last CTA in order
    __shared__ double w1[4], w2[4];
    __shared__ int last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int m = 16; m >= 1; m >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, m);
        s2 += __shfl_xor_sync(0xffffffffu, s2, m);
    }
    if (lane == 0) { w1[wid] = s1; w2[wid] = s2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { a += w1[i]; b += w2[i]; }
        S.part[2 * blockIdx.x] = a;
        S.part[2 * blockIdx.x + 1] = b;
        __threadfence();
        last = atomicAdd(S.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double a = 0.0, b = 0.0;
        for (unsigned c = 0; c < gridDim.x; ++c) {
            a += __ldcg(&S.part[2 * c]);
            b += __ldcg(&S.part[2 * c + 1]);
        }
        S.total[0] = a;
        S.total[1] = b;
        *S.ticket = 0u;
    }
}

// Host scaling of the pattern (rasmussenScaleAB's scaleABInit, :32-61):
// alternating column and row passes in float, in index order.
void scale_init(int n, const std::vector<int>& rptr, const std::vector<int>& col, const std::vector<int>& cptr,
                const std::vector<int>& row, std::vector<float>& rv, std::vector<float>& cv)
{
    rv.assign(n, 1.0f);
    cv.assign(n, 1.0f);
    for (int it = 0; it < kInitialBeta; ++it) {
        for (int j = 0; j < n; ++j) {
            volatile float s = 0.0f;
            for (int q = cptr[j]; q < cptr[j + 1]; ++q) s = s + rv[row[q]];
            cv[j] = 1.0f / s;
        }
        for (int i = 0; i < n; ++i) {
            volatile float s = 0.0f;
            for (int p = rptr[i]; p < rptr[i + 1]; ++p) s = s + cv[col[p]];
            rv[i] = 1.0f / s;
        }
    }
}

int run(const int* cptrs, const int* rows, int n, unsigned long long first, unsigned long long count,
        unsigned long long seed, const spb_options* opt_in, spb_result* out, double* h_per_sample)
{
    const double t0 = wall_seconds();
    if (out) std::memset(out, 0, sizeof(*out));
    if (!cptrs || n < 1 || n > (1 << 20) || count == 0) {
        spb_set_error("approximate permanent: needs column pointers, 1 <= n <= 2^20 and count >= 1");
        if (out) out->status = SPB_ERR_INVALID;
        return SPB_ERR_INVALID;
    }
    const int nnz = cptrs[n];
    if (cptrs[0] != 0 || nnz < 0 || (nnz > 0 && !rows)) {
        spb_set_error("approximate permanent: malformed compressed-column arrays");
        if (out) out->status = SPB_ERR_INVALID;
        return SPB_ERR_INVALID;
    }
    for (int c = 0; c < n; ++c)
        if (cptrs[c + 1] < cptrs[c]) {
            spb_set_error("approximate permanent: column pointers decrease at column %d", c);
            if (out) out->status = SPB_ERR_INVALID;
            return SPB_ERR_INVALID;
        }
    for (int p = 0; p < nnz; ++p)
        if (rows[p] < 0 || rows[p] >= n) {
            spb_set_error("approximate permanent: row index %d out of range", rows[p]);
            if (out) out->status = SPB_ERR_INVALID;
            return SPB_ERR_INVALID;
        }
    // pattern in both orientations (duplicates collapse to one entry)
    std::vector<std::vector<int>> by_row(n);
    std::vector<int> cptr(n + 1, 0), row;
    for (int c = 0; c < n; ++c) {
        std::vector<int> rs(rows + cptrs[c], rows + cptrs[c + 1]);
        std::sort(rs.begin(), rs.end());
        rs.erase(std::unique(rs.begin(), rs.end()), rs.end());
        for (int r : rs) {
            row.push_back(r);
            by_row[r].push_back(c);
        }
        cptr[c + 1] = (int)row.size();
    }
    std::vector<int> rptr(n + 1, 0), col;
    for (int r = 0; r < n; ++r) {
        col.insert(col.end(), by_row[r].begin(), by_row[r].end());
        rptr[r + 1] = (int)col.size();
    }
    std::vector<float> rv, cv;
    scale_init(n, rptr, col, cptr, row, rv, cv);

    spb_options opt;
    if (opt_in) opt = *opt_in; else spb_default_options(&opt);
    int st = SPB_OK;
    DeviceContext* ctx = get_context(opt.device, &st);
    if (!ctx) {
        if (out) out->status = st;
        return st;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    SPB_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t stream = call_stream(ctx, &opt);

    // Launch shape: 8 CTAs of 128 threads per SM (the sampler is latency-bound;
    // 64 registers a thread let all of them be resident), fewer when the per-thread
    // state (5n words) would pass 2 GB or there are fewer samples.
    const int threads = 128;
    unsigned long long T = (unsigned long long)ctx->sm_count * 8 * threads;
    const unsigned long long cap = (2ull << 30) / (20ull * (unsigned long long)n);
    if (T > cap) T = cap;
    if (T > count) T = count;
    int blocks = (int)((T + threads - 1) / threads);
    if (opt.blocks > 0) blocks = opt.blocks;
    if (blocks < 1) blocks = 1;
    T = (unsigned long long)blocks * threads;

    const size_t nn = (size_t)n, nz = (size_t)(nnz > 0 ? row.size() : 1);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + bytes, 256); return o; };
    const size_t o_rp = take(sizeof(int) * (nn + 1)), o_cl = take(sizeof(int) * nz);
    const size_t o_cp = take(sizeof(int) * (nn + 1)), o_rw = take(sizeof(int) * nz);
    const size_t o_r0 = take(sizeof(float) * nn), o_c0 = take(sizeof(float) * nn);
    const size_t o_rv = take(sizeof(float) * nn * T), o_cv = take(sizeof(float) * nn * T);
    const size_t o_re = take(sizeof(int) * nn * T), o_ce = take(sizeof(int) * nn * T);
    const size_t o_sk = take(sizeof(int) * nn * T);
    const size_t o_pt = take(sizeof(double) * 2 * blocks), o_tk = take(sizeof(unsigned) * 4);
    const size_t o_tt = take(sizeof(double) * 2);
    const size_t o_ps = h_per_sample ? take(sizeof(double) * count) : 0;
    if ((st = ensure_scratch(ctx, off)) != SPB_OK) {
        if (out) out->status = st;
        return st;
    }
    char* base = static_cast<char*>(ctx->scratch);
    Pattern P{n,
              reinterpret_cast<int*>(base + o_rp), reinterpret_cast<int*>(base + o_cl),
              reinterpret_cast<int*>(base + o_cp), reinterpret_cast<int*>(base + o_rw),
              reinterpret_cast<float*>(base + o_r0), reinterpret_cast<float*>(base + o_c0)};
    Lane L{reinterpret_cast<float*>(base + o_rv), reinterpret_cast<float*>(base + o_cv),
           reinterpret_cast<int*>(base + o_re), reinterpret_cast<int*>(base + o_ce),
           reinterpret_cast<int*>(base + o_sk), 0, 0};
    Sums S{reinterpret_cast<double*>(base + o_pt), reinterpret_cast<unsigned*>(base + o_tk),
           reinterpret_cast<double*>(base + o_tt), h_per_sample ? reinterpret_cast<double*>(base + o_ps) : nullptr};
    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_call0, stream));
    SPB_CUDA_TRY(cudaMemcpyAsync(base + o_rp, rptr.data(), sizeof(int) * (nn + 1), cudaMemcpyHostToDevice, stream));
    SPB_CUDA_TRY(cudaMemcpyAsync(base + o_cp, cptr.data(), sizeof(int) * (nn + 1), cudaMemcpyHostToDevice, stream));
    if (!row.empty()) {
        SPB_CUDA_TRY(cudaMemcpyAsync(base + o_cl, col.data(), sizeof(int) * col.size(), cudaMemcpyHostToDevice, stream));
        SPB_CUDA_TRY(cudaMemcpyAsync(base + o_rw, row.data(), sizeof(int) * row.size(), cudaMemcpyHostToDevice, stream));
    }
    SPB_CUDA_TRY(cudaMemcpyAsync(base + o_r0, rv.data(), sizeof(float) * nn, cudaMemcpyHostToDevice, stream));
    SPB_CUDA_TRY(cudaMemcpyAsync(base + o_c0, cv.data(), sizeof(float) * nn, cudaMemcpyHostToDevice, stream));
    SPB_CUDA_TRY(cudaMemsetAsync(S.ticket, 0, sizeof(unsigned) * 4, stream));
    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_begin, stream));
    rasmussen_kernel<<<blocks, threads, 0, stream>>>(P, L, first, count, seed, S);
    SPB_CUDA_TRY(cudaGetLastError());
    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_end, stream));
    double tot[2] = {0.0, 0.0};
    SPB_CUDA_TRY(cudaMemcpyAsync(tot, S.total, sizeof(tot), cudaMemcpyDeviceToHost, stream));
    if (h_per_sample)
        SPB_CUDA_TRY(cudaMemcpyAsync(h_per_sample, S.per_sample, sizeof(double) * count, cudaMemcpyDeviceToHost,
                                     stream));
    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_call1, stream));
    SPB_CUDA_TRY(cudaStreamSynchronize(stream));
    if (out) {
        float ms = 0.f, ms_call = 0.f;
        SPB_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev_begin, ctx->ev_end));
        SPB_CUDA_TRY(cudaEventElapsedTime(&ms_call, ctx->ev_call0, ctx->ev_call1));
        const double c = (double)count, mean = tot[0] / c;
        const double var = count > 1 ? (tot[1] - c * mean * mean) / (c - 1.0) : 0.0;
        out->value = mean;
        out->err_est = mean != 0.0 ? std::sqrt(var > 0.0 ? var / c : 0.0) / std::fabs(mean) : INFINITY;
        out->kernel_s = ms * 1e-3;
        out->device_s = ms_call * 1e-3;
        out->gray_steps = count;  // samples
        out->launches = 1;
        out->active_rows = n;
        out->status = SPB_OK;
        out->elapsed_s = wall_seconds() - t0;
    }
    return SPB_OK;
}

}  // namespace approx
}  // namespace spb

extern "C" int spb_perm_approx(const int* cptrs, const int* rows, int n, uint64_t samples, uint64_t seed,
                               const spb_options* opt, spb_result* out)
{
    if (!out) {
        spb_set_error("null result pointer");
        return SPB_ERR_INVALID;
    }
    return spb::approx::run(cptrs, rows, n, 0, samples, seed, opt, out, nullptr);
}

extern "C" int spb_approx_samples(const int* cptrs, const int* rows, int n, uint64_t first, uint64_t count,
                                  uint64_t seed, double* estimates)
{
    if (!estimates) {
        spb_set_error("spb_approx_samples: null output");
        return SPB_ERR_INVALID;
    }
    spb_result r;
    return spb::approx::run(cptrs, rows, n, first, count, seed, nullptr, &r, estimates);
}
