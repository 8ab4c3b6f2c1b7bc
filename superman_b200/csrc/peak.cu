// Pipe-throughput microbenchmarks used as roofline denominators: the FP64
// FMA pipe (dense real/complex/sparse walks) and the integer multiply-add
// pipe (0/1 exact walk).  Each thread runs 8 independent dependency chains so
// the pipe, not latency, bounds the loop.
#include <cuda_runtime.h>

#include "context.h"
#include "spb_common.cuh"

namespace {

__global__ void __launch_bounds__(256) dfma_loop(double* out, int iters, double b, double c)
{
    double a0 = threadIdx.x * 1e-3, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
    double a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
#pragma unroll 1
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a0 = __fma_rn(a0, b, c); a1 = __fma_rn(a1, b, c);
            a2 = __fma_rn(a2, b, c); a3 = __fma_rn(a3, b, c);
            a4 = __fma_rn(a4, b, c); a5 = __fma_rn(a5, b, c);
            a6 = __fma_rn(a6, b, c); a7 = __fma_rn(a7, b, c);
        }
    }
    double s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == 1.2345) out[threadIdx.x] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) imad_loop(unsigned* out, int iters, unsigned b, unsigned c)
{
    unsigned a0 = threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
    unsigned a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
#pragma unroll 1
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a0 = a0 * b + c; a1 = a1 * b + c; a2 = a2 * b + c; a3 = a3 * b + c;
            a4 = a4 * b + c; a5 = a5 * b + c; a6 = a6 * b + c; a7 = a7 * b + c;
        }
    }
    unsigned s = ((a0 ^ a1) + (a2 ^ a3)) + ((a4 ^ a5) + (a6 ^ a7));
    if (s == 0x12345u) out[threadIdx.x] = s;
}

}  // namespace

extern "C" int spb_measure_pipe_peak(int device, int which, double* ops_per_s)
{
    if (!ops_per_s || (which != 0 && which != 1)) {
        spb_set_error("spb_measure_pipe_peak: which must be 0 (fp64 fma) or 1 (int32 mad)");
        return SPB_ERR_INVALID;
    }
    int st = SPB_OK;
    spb::DeviceContext* ctx = spb::get_context(device, &st);
    if (!ctx) return st;
    std::lock_guard<std::mutex> lk(ctx->mu);
    SPB_CUDA_TRY(cudaSetDevice(ctx->device));
    if ((st = spb::ensure_scratch(ctx, 4096)) != SPB_OK) return st;
    const int blocks = ctx->sm_count * 8, threads = 256, iters = 4096;
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        SPB_CUDA_TRY(cudaEventRecord(ctx->ev_begin, ctx->stream));
        if (which == 0)
            dfma_loop<<<blocks, threads, 0, ctx->stream>>>(static_cast<double*>(ctx->scratch), iters, 0.999999, 1e-7);
        else
            imad_loop<<<blocks, threads, 0, ctx->stream>>>(static_cast<unsigned*>(ctx->scratch), iters, 1664525u, 1013904223u);
        SPB_CUDA_TRY(cudaGetLastError());
        SPB_CUDA_TRY(cudaEventRecord(ctx->ev_end, ctx->stream));
        SPB_CUDA_TRY(cudaEventSynchronize(ctx->ev_end));
        float ms = 0.f;
        SPB_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev_begin, ctx->ev_end));
        double ops = (double)blocks * threads * iters * 16.0 * 8.0;
        double rate = ops / (ms * 1e-3);
        if (rep > 0 && rate > best) best = rate;  // first launch is warm-up
    }
    *ops_per_s = best;
    return SPB_OK;
}
