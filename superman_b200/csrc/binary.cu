// Host driver of the exact 0/1 permanent (see binary_impl.cuh).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "binary_impl.cuh"
#include "context.h"

namespace spb {
namespace binary {

// log2 of the Bregman-Minc bound prod_i (r_i!)^(1/r_i) over rows or columns,
// whichever is smaller (an upper bound on the permanent of a 0/1 matrix).
static double log2_perm_bound(const uint8_t* a, int n)
{
    auto side = [&](bool rows) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) {
            int r = 0;
            for (int j = 0; j < n; ++j) r += (rows ? a[i * n + j] : a[j * n + i]) ? 1 : 0;
            if (r == 0) return -HUGE_VAL;
            s += std::lgamma((double)r + 1.0) / std::log(2.0) / r;
        }
        return s;
    };
    return std::fmin(side(true), side(false));
}

// Limbs for the NW sum Sigma = 2^(n-1) perm: |Sigma| < 2^(32L-1).
static int pick_limbs(double perm_bits, int n)
{
    const double bits = perm_bits + (n - 1) + 2;
    if (bits <= 128) return 4;
    if (bits <= 160) return 5;
    if (bits <= 192) return 6;
    if (bits <= 320) return 10;
    return 12;
}

static int run(const uint8_t* a, int n, const spb_options* opt_in, uint32_t* limbs_out,
               spb_result* out)
{
    double t_start = wall_seconds();
    if (!out || !limbs_out) {
        spb_set_error("spb_perm_binary: null output pointer");
        return SPB_ERR_INVALID;
    }
    std::memset(out, 0, sizeof(*out));
    std::memset(limbs_out, 0, sizeof(uint32_t) * 10);
    spb_options opt;
    if (opt_in) opt = *opt_in; else spb_default_options(&opt);
    if (!a || n < 1 || n > kMaxN) {
        spb_set_error("binary permanent needs a non-null matrix and 1 <= n <= %d (got n=%d)", kMaxN, n);
        return out->status = SPB_ERR_INVALID;
    }
    out->gray_steps = (uint64_t)n << (n - 1);
    if (n <= 2) {  // fewer than two walk columns: direct
        const unsigned v = n == 1 ? (a[0] ? 1u : 0u)
                                  : (unsigned)((a[0] && a[3]) ? 1 : 0) + ((a[1] && a[2]) ? 1 : 0);
        limbs_out[0] = v;
        out->value = (double)v;
        out->elapsed_s = wall_seconds() - t_start;
        return out->status = SPB_OK;
    }
    int st = SPB_OK;
    DeviceContext* ctx = get_context(opt.device, &st);
    if (!ctx) return out->status = st;
    std::lock_guard<std::mutex> lk(ctx->mu);
    SPB_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t stream = call_stream(ctx, &opt);

    Problem pb{};
    pb.n = n;
    const double bits = log2_perm_bound(a, n);
    pb.limbs = pick_limbs(bits < 0 ? 0.0 : bits, n);
    // the NW walk runs over the n-1 columns other than the last
    int w = opt.unit_bits > 0 ? opt.unit_bits : 8;
    if (opt.unit_bits <= 0)
        while (w > 2 && (((size_t)1 << w) * n * 4 > 32 * 1024 || n - 1 - w < 16)) --w;
    if (w > 12) w = 12;
    if (w > n - 1) w = n - 1;
    if (w < 2) w = 2;
    pb.w = w;
    pb.units = 1ull << (n - 1 - w);
    const int terms = 1 << w, ntop = n - 1 - w;

    const int tmax = bin_max_threads(n, pb.limbs);
    int threads = opt.threads_per_block > 0 ? (opt.threads_per_block / 32) * 32 : tmax;
    if (threads > tmax) threads = tmax;
    if (threads < 32) threads = 32;
    const size_t smem = sizeof(int) * terms * n + align_up((size_t)(ntop > 0 ? ntop : 1) * n, 16);
    // Default grid: every CTA that fits resident at once (two per SM where
    // the registers allow, e.g. 256 threads at 128 registers).
    int blocks = opt.blocks;
    if (blocks <= 0) {
        int per_sm = 0;
        if ((st = launch_binary(pb, 0, threads, smem, stream, &per_sm)) != SPB_OK) return out->status = st;
        blocks = ctx->sm_count * (per_sm > 0 ? per_sm : 1);
    }
    unsigned long long max_blocks = (pb.units + threads - 1) / threads;
    if ((unsigned long long)blocks > max_blocks) blocks = (int)max_blocks;
    if (blocks < 1) blocks = 1;
    pb.grid = blocks;

    // host-built tables: x'_r = 2 a_{r,n-1} - rowsum_r, doubled low-column
    // counts, doubled high columns
    std::vector<int> x0(n);
    for (int r = 0; r < n; ++r) {
        int rs = 0;
        for (int j = 0; j < n; ++j) rs += a[r * n + j] ? 1 : 0;
        x0[r] = 2 * (a[r * n + n - 1] ? 1 : 0) - rs;
    }
    std::vector<int> dei((size_t)terms * n);
    for (int d = 0; d < terms; ++d)
        for (int r = 0; r < n; ++r) {
            int c = 0;
            for (int j = 0; j < w; ++j) c += ((d >> j) & 1) && a[r * n + j] ? 2 : 0;
            dei[((size_t)(d / 4) * n + r) * 4 + (d % 4)] = c;
        }
    std::vector<int8_t> mt((size_t)(ntop > 0 ? ntop : 1) * n, 0);
    for (int j = 0; j < ntop; ++j)
        for (int r = 0; r < n; ++r) mt[(size_t)j * n + r] = a[r * n + w + j] ? 2 : 0;

    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    const size_t o_x0 = take(sizeof(int) * n);
    const size_t o_de = take(sizeof(int) * dei.size());
    const size_t o_mt = take(mt.size());
    const size_t o_part = take(sizeof(uint32_t) * kMaxLimbs * blocks);
    const size_t o_tick = take(sizeof(unsigned) * 4);
    const size_t o_res = take(sizeof(uint32_t) * kMaxLimbs);
    if ((st = ensure_scratch(ctx, off)) != SPB_OK) return out->status = st;
    char* base = static_cast<char*>(ctx->scratch);
    pb.x0 = reinterpret_cast<const int*>(base + o_x0);
    pb.dei = reinterpret_cast<const int*>(base + o_de);
    pb.mt = reinterpret_cast<const int8_t*>(base + o_mt);
    pb.partials = reinterpret_cast<uint32_t*>(base + o_part);
    pb.ticket = reinterpret_cast<unsigned*>(base + o_tick);
    pb.result = reinterpret_cast<uint32_t*>(base + o_res);

    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_call0, stream));
    SPB_CUDA_TRY(cudaMemcpyAsync(base + o_x0, x0.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream));
    SPB_CUDA_TRY(cudaMemcpyAsync(base + o_de, dei.data(), sizeof(int) * dei.size(), cudaMemcpyHostToDevice, stream));
    SPB_CUDA_TRY(cudaMemcpyAsync(base + o_mt, mt.data(), mt.size(), cudaMemcpyHostToDevice, stream));
    SPB_CUDA_TRY(cudaMemsetAsync(pb.ticket, 0, sizeof(unsigned) * 4, stream));
    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_begin, stream));
    if ((st = launch_binary(pb, blocks, threads, smem, stream)) != SPB_OK) return out->status = st;
    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_end, stream));
    uint32_t res[kMaxLimbs] = {0};
    SPB_CUDA_TRY(cudaMemcpyAsync(res, pb.result, sizeof(uint32_t) * pb.limbs, cudaMemcpyDeviceToHost, stream));
    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_call1, stream));
    SPB_CUDA_TRY(cudaStreamSynchronize(stream));
    float ms = 0.f, ms_call = 0.f;
    SPB_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev_begin, ctx->ev_end));
    SPB_CUDA_TRY(cudaEventElapsedTime(&ms_call, ctx->ev_call0, ctx->ev_call1));

    const int L = pb.limbs;
    if (!(n & 1)) {  // perm = (+-) Sigma / 2^(n-1), + for odd n: negate mod 2^(32L)
        uint64_t c = 1;
        for (int l = 0; l < L; ++l) {
            uint64_t t = (uint64_t)(~res[l]) + c;
            res[l] = (uint32_t)t;
            c = t >> 32;
        }
    }
    // arithmetic shift right by n-1 bits (Sigma is a multiple of 2^(n-1))
    const bool neg = (res[L - 1] >> 31) & 1u;
    uint32_t ext[kMaxLimbs + 2];
    for (int l = 0; l < kMaxLimbs + 2; ++l) ext[l] = l < L ? res[l] : (neg ? 0xffffffffu : 0u);
    const int sh = n - 1, ws = sh / 32, bs = sh % 32;
    uint32_t shifted[kMaxLimbs];
    for (int l = 0; l < kMaxLimbs; ++l) {
        const uint32_t lo = l + ws < kMaxLimbs + 2 ? ext[l + ws] : (neg ? 0xffffffffu : 0u);
        const uint32_t hi = l + ws + 1 < kMaxLimbs + 2 ? ext[l + ws + 1] : (neg ? 0xffffffffu : 0u);
        shifted[l] = bs ? (lo >> bs) | (hi << (32 - bs)) : lo;
    }
    constexpr int kOutLimbs = 10;  // the C ABI's 320-bit result
    for (int l = 0; l < kOutLimbs; ++l) limbs_out[l] = shifted[l];
    // double approximation of the signed integer
    double v = 0.0;
    uint32_t mag[kOutLimbs];
    std::memcpy(mag, limbs_out, sizeof(mag));
    if (neg) {
        uint64_t c = 1;
        for (int l = 0; l < kOutLimbs; ++l) {
            uint64_t t = (uint64_t)(~mag[l]) + c;
            mag[l] = (uint32_t)t;
            c = t >> 32;
        }
    }
    for (int l = kOutLimbs - 1; l >= 0; --l) v = v * 4294967296.0 + (double)mag[l];
    out->value = neg ? -v : v;
    out->kernel_s = ms * 1e-3;
    out->device_s = ms_call * 1e-3;
    out->launches = 1;
    out->elapsed_s = wall_seconds() - t_start;
    return out->status = SPB_OK;
}

}  // namespace binary
}  // namespace spb

extern "C" int spb_perm_binary(const uint8_t* a, int n, const spb_options* opt, uint32_t* limbs,
                               spb_result* out)
{
    return spb::binary::run(a, n, opt, limbs, out);
}
