// Library-wide host state: error strings, per-device contexts, scratch arena.
#include "context.h"

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <memory>

#include "spb_common.cuh"

namespace {
thread_local char g_last_error[512] = "";
std::mutex g_ctx_mu;
std::unique_ptr<spb::DeviceContext> g_ctx[64];
}  // namespace

void spb_set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

extern "C" const char* spb_last_error(void) { return g_last_error; }

extern "C" const char* spb_status_string(int status)
{
    switch (status) {
    case SPB_OK: return "ok";
    case SPB_ERR_INVALID: return "invalid argument";
    case SPB_ERR_CUDA: return "cuda error";
    case SPB_ERR_NO_DEVICE: return "no cuda device";
    case SPB_ERR_OOM: return "out of memory";
    case SPB_ERR_OVERFLOW: return "result overflow";
    case SPB_ERR_TIMEOUT: return "timeout";
    case SPB_ERR_CANCELLED: return "cancelled";
    case SPB_ERR_BUSY: return "busy";
    case SPB_ERR_IO: return "io error";
    case SPB_ERR_NOT_SQUARE: return "matrix is not square";
    case SPB_ERR_ACCURACY: return "estimated error above the bound";
    default: return "unknown status";
    }
}

extern "C" int spb_version(void) { return 100; }

extern "C" int spb_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

extern "C" void spb_default_options(spb_options* opt)
{
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->device = 0;
    opt->precision = SPB_PREC_FP64;
    opt->rel_tol = 0.0;
}

namespace spb {

DeviceContext* get_context(int device, int* st)
{
    *st = SPB_OK;
    if (device < 0 || device >= 64) {
        spb_set_error("device ordinal %d out of range", device);
        *st = SPB_ERR_INVALID;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (g_ctx[device]) return g_ctx[device].get();
    int count = spb_device_count();
    if (device >= count) {
        spb_set_error("no CUDA device %d (%d visible)", device, count);
        *st = SPB_ERR_NO_DEVICE;
        return nullptr;
    }
    std::unique_ptr<DeviceContext> ctx(create_context(device, st));
    if (!ctx) return nullptr;
    g_ctx[device] = std::move(ctx);
    return g_ctx[device].get();
}

DeviceContext* create_context(int device, int* st)
{
    *st = SPB_OK;
    auto ctx = std::make_unique<DeviceContext>();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    int optin = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_begin);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_end);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_call0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_call1);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_ref0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_ref1);
    if (e != cudaSuccess) {
        spb_set_error("device %d init failed: %s", device, cudaGetErrorString(e));
        *st = SPB_ERR_CUDA;
        destroy_context(ctx.release());
        return nullptr;
    }
    // Dynamic shared memory budget for the walk kernels: the opt-in limit less
    // a reserve for their static shared arrays (reductions, flags).
    ctx->smem_optin = optin > 4096 ? (size_t)optin - 4096 : (size_t)optin;
    return ctx.release();
}

void destroy_context(DeviceContext* ctx)
{
    if (!ctx) return;
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->release_small_graphs) ctx->release_small_graphs(ctx->small_graphs);
    for (cudaEvent_t ev : {ctx->ev_begin, ctx->ev_end, ctx->ev_call0, ctx->ev_call1, ctx->ev_ref0, ctx->ev_ref1})
        if (ev) cudaEventDestroy(ev);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->list) cudaFree(ctx->list);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

// Allocation failures injected by spb_debug_fail_allocations: each of the
// next g_fail_allocs calls of ensure_scratch / ensure_list / ensure_pinned
// reports SPB_ERR_OOM without allocating (or freeing) anything.
static std::atomic<int> g_fail_allocs{0};

bool injected_failure(const char* what)
{
    int k = g_fail_allocs.load();
    while (k > 0 && !g_fail_allocs.compare_exchange_weak(k, k - 1)) {
    }
    if (k <= 0) return false;
    spb_set_error("%s: allocation failure injected for testing", what);
    return true;
}

int ensure_scratch(DeviceContext* ctx, size_t bytes)
{
    if (injected_failure("scratch")) return SPB_ERR_OOM;
    if (bytes <= ctx->scratch_bytes) return SPB_OK;
    if (ctx->scratch) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
    }
    size_t want = align_up(bytes < (1u << 20) ? (1u << 20) : bytes, 1u << 20);
    if (cudaMalloc(&ctx->scratch, want) != cudaSuccess) {
        cudaGetLastError();
        spb_set_error("cudaMalloc of %zu scratch bytes failed", want);
        return SPB_ERR_OOM;
    }
    ctx->scratch_bytes = want;
    return SPB_OK;
}

int ensure_list(DeviceContext* ctx, size_t bytes)
{
    if (injected_failure("refinement list")) return SPB_ERR_OOM;
    if (bytes <= ctx->list_bytes) return SPB_OK;
    if (ctx->list) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->list);
        ctx->list = nullptr;
        ctx->list_bytes = 0;
    }
    size_t want = align_up(bytes, 1u << 20);
    if (cudaMalloc(&ctx->list, want) != cudaSuccess) {
        cudaGetLastError();
        spb_set_error("cudaMalloc of %zu refinement-list bytes failed", want);
        return SPB_ERR_OOM;
    }
    ctx->list_bytes = want;
    return SPB_OK;
}

int ensure_pinned(DeviceContext* ctx, size_t bytes)
{
    if (injected_failure("pinned")) return SPB_ERR_OOM;
    if (bytes <= ctx->pinned_bytes) return SPB_OK;
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_dev = nullptr;
    ctx->pinned_bytes = 0;
    size_t want = align_up(bytes < (1u << 16) ? (1u << 16) : bytes, 1u << 16);
    if (cudaMallocHost(&ctx->pinned, want) != cudaSuccess) {
        cudaGetLastError();
        spb_set_error("cudaMallocHost of %zu bytes failed", want);
        return SPB_ERR_OOM;
    }
    ctx->pinned_bytes = want;
    // page-locked memory is mapped into the device's address space under
    // unified addressing; kernels may then write results straight into it
    if (cudaHostGetDevicePointer(&ctx->pinned_dev, ctx->pinned, 0) != cudaSuccess) {
        cudaGetLastError();
        ctx->pinned_dev = nullptr;
    }
    return SPB_OK;
}

}  // namespace spb

extern "C" void spb_debug_fail_allocations(int count) { spb::g_fail_allocs.store(count > 0 ? count : 0); }
