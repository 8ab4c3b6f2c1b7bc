// Many small permanents in one launch: one warp per matrix.
//
// The whole-GPU walk (dense_impl.cuh) spreads one permanent over every SM;
// for n <= 24 a permanent is too small for that (2^(n-1) terms, a few
// microseconds of FP64 work) and launch latency dominates.  Here each warp
// takes a matrix of the batch (grid-stride over the batch), builds its row
// scaling, double-double NW start vector, low-column subset-sum table and
// high columns in the warp's slice of shared memory, then its 32 lanes split
// the Gray units of that matrix exactly as the threads of the big walk do
// (same unit evaluators; the double-double unit bases live in registers), and
// a warp reduction gives the double-double total.  The permanent of matrix m
// is written as (hi, lo) per component: out[m*2*comps + 2*c + {0, 1}].
//
// Device pointers only, no allocation, no host synchronisation: the serving
// loop captures one launch per batch shape in a CUDA graph, and the
// decomposition path runs its independent pieces through it.
#include <cuda_runtime.h>

#include "batch.h"
#include "dense_impl.cuh"
#include "spb_common.cuh"

namespace spb {
namespace batch {

constexpr int kWarpsPerCta = 4;

template <int N, int C>
struct Cfg {
    static constexpr int W = (N - 1) < 5 ? (N - 1) : 5;  // low column bits per unit
    static constexpr int G = C == 1 ? (W >= 2 ? 4 : (W == 1 ? 2 : 1)) : (W >= 1 ? 2 : 1);
    static constexpr int TERMS = 1 << W;
    static constexpr int NTOP = N - 1 - W;
    static constexpr int NTP = NTOP > 0 ? NTOP : 0;
    // Unit-base lo words: registers, except complex n >= 21, where hi and lo
    // of both parts (4n doubles) would spill; there they sit in a lane-private
    // slot of the warp's shared slice.  (With 32 terms per unit the slot's
    // per-unit traffic costs more than it saves wherever registers suffice.)
    static constexpr bool LO_SMEM = C == 2 && N >= 21;
    static constexpr int LO_DOUBLES = LO_SMEM ? 32 * N * C : 0;
    // doubles per warp: DE table, high columns, x0 hi/lo, lo words, row
    // exponents (as doubles), rounded up to 32 bytes: the unit evaluator reads
    // the DE table with 16-byte vector loads, so every warp's slice must start
    // aligned.
    static constexpr int SMEM_DOUBLES = (TERMS * N * C + NTP * N * C + 2 * N * C + LO_DOUBLES + N + 3) / 4 * 4;
    static_assert(SMEM_DOUBLES % 4 == 0, "per-warp shared slice must keep 32-byte alignment");
};

// Matrix m of a batch starts at mats + m*N*N*C, or, with an offset table, at
// mats + offs[m] * kOffsetUnit doubles (the serving loop's device pool).

// With `src` (the serving loop's page-locked host mirror, mapped into the
// device's address space, at the same offsets), each warp first copies its
// matrix from src into its place in mats, so every matrix crosses the host
// link once, in coalesced reads that overlap the other warps' work.
template <int N, int C>
__global__ void __launch_bounds__(kWarpsPerCta * 32) batch_walk(double* __restrict__ mats,
                                                                 const unsigned* __restrict__ offs,
                                                                 const double* __restrict__ src,
                                                                 int count, double* __restrict__ out)
{
    using Q = Cfg<N, C>;
    constexpr int G = Q::G, TERMS = Q::TERMS, NTOP = Q::NTOP, NTP = Q::NTP, W = Q::W;
    extern __shared__ __align__(16) double smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double* s_de = smem + (size_t)wid * Q::SMEM_DOUBLES;  // [C][TERMS/G][N][G]
    double* s_mt = s_de + TERMS * N * C;                  // [C][NTOP][N]
    double* s_x0h = s_mt + NTP * N * C;                   // [C][N]
    double* s_x0l = s_x0h + N * C;                        // [C][N]
    double* s_lo = s_x0l + N * C;                         // [C][N][32] lane-private lo words (LO_SMEM)
    int* s_exp = reinterpret_cast<int*>(s_lo + Q::LO_DOUBLES);  // [N]

    const int total_warps = gridDim.x * kWarpsPerCta;
    for (int m = blockIdx.x * kWarpsPerCta + wid; m < count; m += total_warps) {
        const size_t base = offs ? (size_t)offs[m] * kOffsetUnit : (size_t)m * N * N * C;
        if (src) {
            for (int i = lane; i < N * N * C; i += 32) mats[base + i] = src[base + i];
            __syncwarp();  // orders the warp's writes before its reads below
        }
        const double* A = mats + base;
        // row exponents: row max scaled into [0.5, 1)
        for (int r = lane; r < N; r += 32) {
            double mx = 0.0;
            for (int j = 0; j < N * C; ++j) mx = fmax(mx, fabs(A[r * N * C + j]));
            int e = 0;
            if (mx > 0.0 && isfinite(mx)) frexp(mx, &e);
            s_exp[r] = e;
        }
        __syncwarp();
        // NW start vector (double-double)
        for (int rr = lane; rr < N * C; rr += 32) {
            const int r = rr / C, part = rr % C;
            dd s = {0.0, 0.0};
            for (int j = 0; j < N; ++j) s = dd_add_d(s, ldexp(A[(r * N + j) * C + part], -s_exp[r]));
            dd h = {-0.5 * s.hi, -0.5 * s.lo};
            dd x = dd_add_d(h, ldexp(A[(r * N + (N - 1)) * C + part], -s_exp[r]));
            s_x0h[part * N + r] = x.hi;
            s_x0l[part * N + r] = x.lo;
        }
        // low-column subset sums, grouped [part][d/G][r][d%G]
        for (int idx = lane; idx < TERMS * N * C; idx += 32) {
            const int part = idx / (TERMS * N), rem = idx % (TERMS * N);
            const int d = rem / N, r = rem % N;
            dd s = {0.0, 0.0};
            for (int j = 0; j < W; ++j)
                if ((d >> j) & 1) s = dd_add_d(s, ldexp(A[(r * N + j) * C + part], -s_exp[r]));
            s_de[part * TERMS * N + ((d / G) * N + r) * G + (d % G)] = s.hi;
        }
        // high columns [part][j][r]
        if constexpr (NTP > 0)
            for (int idx = lane; idx < NTP * N * C; idx += 32) {
                const int part = idx / (NTP * N), rem = idx % (NTP * N);
                const int j = rem / N, r = rem % N;
                s_mt[idx] = ldexp(A[(r * N + (W + j)) * C + part], -s_exp[r]);
            }
        __syncwarp();

        unsigned long long u0, u1;
        balanced_range(1ull << NTP, 32, lane, &u0, &u1);
        dd tot[C];
#pragma unroll
        for (int c = 0; c < C; ++c) tot[c] = {0.0, 0.0};
        if (u0 < u1) {
            // unit base: hi words in registers; lo words in registers or in the
            // lane's shared slot (element (c, r) at [(c * N + r) * 32 + lane])
            double xh[C][N];
            double xlr[Q::LO_SMEM ? 1 : C * N];
            double* xl = Q::LO_SMEM ? s_lo + lane : xlr;
            constexpr int LS = Q::LO_SMEM ? 32 : 1;  // stride between elements
            const unsigned long long g0 = gray_of(u0);
#pragma unroll
            for (int c = 0; c < C; ++c)
#pragma unroll
                for (int r = 0; r < N; ++r) {
                    dd x = {s_x0h[c * N + r], s_x0l[c * N + r]};
                    for (int j = 0; j < NTOP; ++j)
                        if ((g0 >> j) & 1ull) x = dd_add_d(x, s_mt[c * NTP * N + j * N + r]);
                    xh[c][r] = x.hi;
                    xl[(c * N + r) * LS] = x.lo;
                }
            unsigned long long u = u0;
            while (true) {
                if constexpr (C == 1) {
                    double us = dense::unit_sum_real<N, G>(xh[0], s_de, TERMS / G);
                    tot[0] = dd_add_d(tot[0], (u & 1ull) ? -us : us);
                } else {
                    double ur, ui;
                    dense::unit_sum_complex<N, G>(xh[0], xh[C - 1], s_de, s_de + TERMS * N, TERMS / G, ur, ui);
                    if (u & 1ull) { ur = -ur; ui = -ui; }
                    tot[0] = dd_add_d(tot[0], ur);
                    tot[C - 1] = dd_add_d(tot[C - 1], ui);
                }
                if (++u >= u1) break;
                const int j = __ffsll((long long)u) - 1;
                const bool add = (gray_of(u) >> j) & 1ull;
#pragma unroll
                for (int c = 0; c < C; ++c)
#pragma unroll
                    for (int r = 0; r < N; ++r) {
                        const double v = s_mt[c * NTP * N + j * N + r];
                        dd s = two_sum(xh[c][r], add ? v : -v);
                        dd z = fast_two_sum(s.hi, add_rn(s.lo, xl[(c * N + r) * LS]));
                        xh[c][r] = z.hi;
                        xl[(c * N + r) * LS] = z.lo;
                    }
            }
        }
#pragma unroll
        for (int c = 0; c < C; ++c) tot[c] = warp_sum_dd(tot[c]);
        if (lane == 0) {
            int es = 0;
            for (int r = 0; r < N; ++r) es += s_exp[r];
            const double sgn = (N % 2) ? 1.0 : -1.0;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                out[(size_t)m * 2 * C + 2 * c] = sgn * ldexp(tot[c].hi, es + 1);
                out[(size_t)m * 2 * C + 2 * c + 1] = sgn * ldexp(tot[c].lo, es + 1);
            }
        }
        __syncwarp();
    }
}

template <int N, int C>
int launch_n(double* mats, const unsigned* offs, const double* src, int count, double* out, int sms,
             cudaStream_t s)
{
    constexpr size_t smem = sizeof(double) * Cfg<N, C>::SMEM_DOUBLES * kWarpsPerCta;
    if (smem > 48 * 1024) {
        static cudaError_t attr = cudaFuncSetAttribute(batch_walk<N, C>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        SPB_CUDA_TRY(attr);
    }
    int blocks = (count + kWarpsPerCta - 1) / kWarpsPerCta;
    const int cap = sms * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    batch_walk<N, C><<<blocks, kWarpsPerCta * 32, smem, s>>>(mats, offs, src, count, out);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

int dispatch(double* mats, const unsigned* offs, const double* src, int n, int is_complex, int count, double* out,
             int sms, cudaStream_t s)
{
    const int key = n * 2 + (is_complex ? 1 : 0);
    switch (key) {
#define SPB_BCASE(N)                                                               \
    case 2 * N: return launch_n<N, 1>(mats, offs, src, count, out, sms, s);        \
    case 2 * N + 1: return launch_n<N, 2>(mats, offs, src, count, out, sms, s);
        SPB_BCASE(1) SPB_BCASE(2) SPB_BCASE(3) SPB_BCASE(4) SPB_BCASE(5) SPB_BCASE(6) SPB_BCASE(7)
        SPB_BCASE(8) SPB_BCASE(9) SPB_BCASE(10) SPB_BCASE(11) SPB_BCASE(12) SPB_BCASE(13)
        SPB_BCASE(14) SPB_BCASE(15) SPB_BCASE(16) SPB_BCASE(17) SPB_BCASE(18) SPB_BCASE(19)
        SPB_BCASE(20) SPB_BCASE(21) SPB_BCASE(22) SPB_BCASE(23) SPB_BCASE(24)
#undef SPB_BCASE
    default:
        spb_set_error("batched walk: unsupported n=%d", n);
        return SPB_ERR_INVALID;
    }
}

int launch_gathered(const double* src, double* dst, const unsigned* d_offs, int n, int is_complex, int count,
                    double* d_out, cudaStream_t s)
{
    if (n < 1 || n > kMaxN || count < 0) {
        spb_set_error("batched walk: n=%d outside 1..%d or negative count", n, kMaxN);
        return SPB_ERR_INVALID;
    }
    if (count == 0) return SPB_OK;
    int dev = 0, sms = 0;
    SPB_CUDA_TRY(cudaGetDevice(&dev));
    SPB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return dispatch(dst, d_offs, src, n, is_complex, count, d_out, sms, s);
}

}  // namespace batch
}  // namespace spb

extern "C" int spb_perm_batch_dev(const double* d_mats, int n, int is_complex, int count, double* d_out,
                                  void* stream)
{
    using namespace spb::batch;
    if (!d_mats || !d_out || count < 0) {
        spb_set_error("spb_perm_batch_dev: null pointer or negative count");
        return SPB_ERR_INVALID;
    }
    if (n < 1 || n > kMaxN) {
        spb_set_error("spb_perm_batch_dev: n=%d outside 1..%d (larger n: the whole-GPU entry points)", n, kMaxN);
        return SPB_ERR_INVALID;
    }
    if (count == 0) return SPB_OK;
    int dev = 0, sms = 0;
    SPB_CUDA_TRY(cudaGetDevice(&dev));
    SPB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the matrices are read in place (the cast drops const: with no source
    // the kernel only reads them)
    return dispatch(const_cast<double*>(d_mats), nullptr, nullptr, n, is_complex, count, d_out, sms, s);
}
