// Per-device runtime state shared by every entry point: a stream, timing
// events, a grow-only device scratch arena and a pinned host staging buffer.
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <mutex>

#include "superman_b200.h"

namespace spb {

struct DeviceContext {
    int device = -1;
    int sm_count = 0;
    size_t smem_optin = 0;  // max dynamic shared memory per block (opt-in)
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;      // around the walk kernels
    cudaEvent_t ev_call0 = nullptr, ev_call1 = nullptr;    // around the whole call
    cudaEvent_t ev_ref0 = nullptr, ev_ref1 = nullptr;      // around the refinement passes
    void* list = nullptr;  // refinement work list (grow-only)
    size_t list_bytes = 0;
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    void* pinned_dev = nullptr;  // the device's address of `pinned` (null if it has none)
    // CUDA graphs of the fused small call, cached per launch (small_call.cu
    // owns the cache; destroy_context frees it through release_small_graphs).
    void* small_graphs = nullptr;
    void (*release_small_graphs)(void*) = nullptr;
    std::mutex mu;  // serialises calls that use this context
};

// Returns the context of `device`, creating it on first use (status in *st).
DeviceContext* get_context(int device, int* st);

// A context owned by the caller (not the device's shared one): its own
// stream, events and arenas, so that calls through it can overlap calls
// through other contexts on the same device.  Free with destroy_context.
DeviceContext* create_context(int device, int* st);
void destroy_context(DeviceContext* ctx);

// Ensures ctx->scratch holds at least `bytes` (grows, never shrinks).
int ensure_scratch(DeviceContext* ctx, size_t bytes);

// Ensures ctx->list holds at least `bytes` (grows, never shrinks).
int ensure_list(DeviceContext* ctx, size_t bytes);

// Ensures ctx->pinned holds at least `bytes` of page-locked host memory.
int ensure_pinned(DeviceContext* ctx, size_t bytes);

// True (and the error message set) when an allocation failure injected by
// spb_debug_fail_allocations is due; every allocation site checks it first.
bool injected_failure(const char* what);

// Resolves the stream to use for a call.
inline cudaStream_t call_stream(DeviceContext* ctx, const spb_options* opt)
{
    return (opt && opt->stream) ? static_cast<cudaStream_t>(opt->stream) : ctx->stream;
}

inline double wall_seconds()
{
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace spb
