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

static int pick_limbs(double bits)
{
    if (bits + 2 <= 128) return 4;
    if (bits + 2 <= 192) return 6;
    return 10;
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
    std::memset(limbs_out, 0, sizeof(uint32_t) * kMaxLimbs);
    spb_options opt;
    if (opt_in) opt = *opt_in; else spb_default_options(&opt);
    if (!a || n < 1 || n > kMaxN) {
        spb_set_error("binary permanent needs a non-null matrix and 1 <= n <= %d (got n=%d)", kMaxN, n);
        return out->status = SPB_ERR_INVALID;
    }
    out->gray_steps = (uint64_t)n << n;
    if (n == 1) {  // no subset walk needed
        limbs_out[0] = a[0] ? 1u : 0u;
        out->value = a[0] ? 1.0 : 0.0;
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
    pb.limbs = pick_limbs(bits < 0 ? 0.0 : bits);
    int w = opt.unit_bits > 0 ? opt.unit_bits : 8;
    if (opt.unit_bits <= 0)
        while (w > 2 && (((size_t)1 << w) * n * 4 > 32 * 1024 || n - w < 16)) --w;
    if (w > 12) w = 12;
    if (w > n) w = n;
    if (w < 2) w = 2;
    pb.w = w;
    pb.units = 1ull << (n - w);
    const int terms = 1 << w, ntop = n - w;

    const int tmax = bin_max_threads(n);
    int threads = opt.threads_per_block > 0 ? (opt.threads_per_block / 32) * 32 : tmax;
    if (threads > tmax) threads = tmax;
    if (threads < 32) threads = 32;
    int blocks = opt.blocks > 0 ? opt.blocks : ctx->sm_count;
    unsigned long long max_blocks = (pb.units + threads - 1) / threads;
    if ((unsigned long long)blocks > max_blocks) blocks = (int)max_blocks;
    if (blocks < 1) blocks = 1;
    pb.grid = blocks;
    const size_t smem = sizeof(int) * terms * n + align_up((size_t)(ntop > 0 ? ntop : 1) * n, 16);

    // host-built tables
    std::vector<int> dei((size_t)terms * n);
    for (int d = 0; d < terms; ++d)
        for (int r = 0; r < n; ++r) {
            int c = 0;
            for (int j = 0; j < w; ++j) c += ((d >> j) & 1) && a[r * n + j] ? 1 : 0;
            dei[((size_t)(d / 4) * n + r) * 4 + (d % 4)] = c;
        }
    std::vector<int8_t> mt((size_t)(ntop > 0 ? ntop : 1) * n, 0);
    for (int j = 0; j < ntop; ++j)
        for (int r = 0; r < n; ++r) mt[(size_t)j * n + r] = a[r * n + w + j] ? 1 : 0;

    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    const size_t o_de = take(sizeof(int) * dei.size());
    const size_t o_mt = take(mt.size());
    const size_t o_part = take(sizeof(uint32_t) * kMaxLimbs * blocks);
    const size_t o_tick = take(sizeof(unsigned) * 4);
    const size_t o_res = take(sizeof(uint32_t) * kMaxLimbs);
    if ((st = ensure_scratch(ctx, off)) != SPB_OK) return out->status = st;
    char* base = static_cast<char*>(ctx->scratch);
    pb.dei = reinterpret_cast<const int*>(base + o_de);
    pb.mt = reinterpret_cast<const int8_t*>(base + o_mt);
    pb.partials = reinterpret_cast<uint32_t*>(base + o_part);
    pb.ticket = reinterpret_cast<unsigned*>(base + o_tick);
    pb.result = reinterpret_cast<uint32_t*>(base + o_res);

    SPB_CUDA_TRY(cudaEventRecord(ctx->ev_call0, stream));
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
    if (n & 1) {  // perm = (-1)^n * sum, negate mod 2^(32L)
        uint64_t c = 1;
        for (int l = 0; l < L; ++l) {
            uint64_t t = (uint64_t)(~res[l]) + c;
            res[l] = (uint32_t)t;
            c = t >> 32;
        }
    }
    const bool neg = (res[L - 1] >> 31) & 1u;
    for (int l = 0; l < kMaxLimbs; ++l) limbs_out[l] = l < L ? res[l] : (neg ? 0xffffffffu : 0u);
    // double approximation of the signed integer
    double v = 0.0;
    uint32_t mag[kMaxLimbs];
    std::memcpy(mag, limbs_out, sizeof(mag));
    if (neg) {
        uint64_t c = 1;
        for (int l = 0; l < kMaxLimbs; ++l) {
            uint64_t t = (uint64_t)(~mag[l]) + c;
            mag[l] = (uint32_t)t;
            c = t >> 32;
        }
    }
    for (int l = kMaxLimbs - 1; l >= 0; --l) v = v * 4294967296.0 + (double)mag[l];
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
