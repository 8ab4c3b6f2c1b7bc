// Dense real permanent that performs no device or host allocation.
//
// Who needs it: callers that cannot let a library call cudaMalloc/cudaFree.
// Typical cases are host programs that reserve all of device memory up front
// for their own pool allocator (a foreign cudaMalloc then fails or fragments
// that pool), and latency-bound request loops that cannot afford cudaFree's
// implicit device-wide synchronisation or an out-of-memory failure in the
// middle of a request.  This entry point takes device pointers for the input
// and the result, launches on the caller's stream, and keeps all of its
// working memory in one fixed file-scope device array.
//
// Precision: the FP64 walk (the allocating entry points' SPB_PREC_FP64: FP64
// row sums and products, double-double sums, no double-double refinement of
// dominant units).  On U[0,1) inputs that is about 1e-13 relative at n=24 and
// 3e-12 at n=32; the error grows with the cancellation of Ryser's sum.
//
// Working memory: g_noalloc_scratch below, kNoAllocScratchBytes (256 KiB) per
// GPU that loads this library, held until the process exits.  It holds the
// row-scaled matrix, the subset-sum tables, the per-CTA partial sums, the
// last-CTA ticket and the grid total, laid out exactly as the allocating
// path lays out its scratch arena.  Sizes up to n = kNoAllocMaxN (40) fit;
// larger n is rejected with SPB_ERR_INVALID.
//
// Sharing: every call on a device uses the same array and leaves its contents
// behind.  The setup kernel of each call zeroes the ticket and counters the
// later kernels accumulate into, and everything else is overwritten before
// it is read.  Two calls whose kernels overlap on the GPU (different streams,
// or different host threads without ordering) race on the array and give
// wrong results; order them on one stream.
//
// Set-up: the first call on each device, with that device current, looks up
// the array's device address with cudaGetSymbolAddress and caches it (the
// symbol name itself is only a host-side stand-in, never a device address),
// and loads every kernel this entry point can launch, setting their
// shared-memory limits.  With CUDA's default lazy module loading the driver
// would otherwise load each kernel, and place the array, on its first launch,
// which can allocate device memory.  So make the first call before reserving
// the rest of device memory for a pool, and before any stream capture.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "dense_impl.cuh"
#include "spb_common.cuh"

namespace spb {
namespace dense {
// Defined in dense.cu.
__global__ void setup_kernel(Problem pb, const double* __restrict__ a_in, int smem_tables);
int launch_setup(const Problem& pb, const double* d_a, cudaStream_t s);
int group_size(int n, int comps);
int choose_unit_bits(int n, int comps, const spb_options* opt);
size_t plan_layout(Problem* pb, char* base, size_t* in_offset);
size_t walk_smem_bytes(const Problem& pb, int threads);
int prepare_setup(int* limit);
int prepare_walk_real(int n);  // dense_dispatch.cu
}  // namespace dense
}  // namespace spb

namespace {

constexpr int kNoAllocMaxN = 40;
constexpr size_t kNoAllocScratchBytes = 256 * 1024;
constexpr int kNoAllocMaxBlocks = 1024;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::once_flag g_once[64];
void* g_scratch_ptr[64];
cudaError_t g_scratch_err[64];
int g_prepare_st[64];

// perm = (4(n%2)-2) * total * 2^E, written as a double-double {hi, lo}.
__global__ void noalloc_finalize(spb::dense::Problem pb, double* out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const int e = *pb.exp_sum + 1;
        const double sgn = (pb.n % 2) ? 1.0 : -1.0;
        out[0] = sgn * ldexp(pb.result[0].hi, e);
        out[1] = sgn * ldexp(pb.result[0].lo, e);
    }
}

// Once per device, with it current: the array's address, then every kernel
// a call can launch (setup_kernel, walk_real<1..kNoAllocMaxN>,
// noalloc_finalize), loaded and configured without launching.
void set_up_device(int dev)
{
    g_scratch_err[dev] = cudaGetSymbolAddress(&g_scratch_ptr[dev], g_noalloc_scratch);
    if (g_scratch_err[dev] != cudaSuccess) return;
    int st = spb::dense::prepare_setup(nullptr);
    for (int n = 1; n <= kNoAllocMaxN && st == SPB_OK; ++n) st = spb::dense::prepare_walk_real(n);
    if (st == SPB_OK) {
        cudaFuncAttributes fa{};
        const cudaError_t e = cudaFuncGetAttributes(&fa, noalloc_finalize);
        if (e != cudaSuccess) {
            spb_set_error("spb_perm_dense_f64_noalloc: loading its kernels failed: %s", cudaGetErrorString(e));
            st = SPB_ERR_CUDA;
        }
    }
    g_prepare_st[dev] = st;
}

}  // namespace

extern "C" int spb_perm_dense_f64_noalloc(const double* d_a, int n, double* d_out, void* stream)
{
    using namespace spb::dense;
    if (!d_a || !d_out) {
        spb_set_error("spb_perm_dense_f64_noalloc: null device pointer");
        return SPB_ERR_INVALID;
    }
    if (n < 1 || n > kNoAllocMaxN) {
        spb_set_error("spb_perm_dense_f64_noalloc: n=%d outside 1..%d (its fixed %zu-byte "
                      "working array holds at most n=%d)", n, kNoAllocMaxN, kNoAllocScratchBytes,
                      kNoAllocMaxN);
        return SPB_ERR_INVALID;
    }
    int dev = 0;
    SPB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        spb_set_error("spb_perm_dense_f64_noalloc: device %d out of range", dev);
        return SPB_ERR_INVALID;
    }
    std::call_once(g_once[dev], [dev] { set_up_device(dev); });
    if (g_scratch_err[dev] != cudaSuccess) {
        spb_set_error("spb_perm_dense_f64_noalloc: cudaGetSymbolAddress failed: %s",
                      cudaGetErrorString(g_scratch_err[dev]));
        return SPB_ERR_CUDA;
    }
    if (g_prepare_st[dev] != SPB_OK) return g_prepare_st[dev];
    int sms = 0, optin = 0;
    SPB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SPB_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t smem_budget = optin > 4096 ? (size_t)optin - 4096 : (size_t)optin;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // Same shape rules as the allocating entry point.
    spb_options opt;
    spb_default_options(&opt);
    Problem pb{};
    pb.n = n;
    pb.na = n;
    pb.comps = 1;
    pb.w = choose_unit_bits(n, 1, &opt);
    pb.g = group_size(n, 1);
    pb.units = 1ull << (n - 1 - pb.w);
    int threads = walk_max_threads(n, 1);
    while (threads > 64 && walk_smem_bytes(pb, threads) > smem_budget) threads -= 32;
    threads = (threads / 32) * 32;
    const size_t smem = walk_smem_bytes(pb, threads);
    if (smem > smem_budget) {
        spb_set_error("spb_perm_dense_f64_noalloc: n=%d needs %zu B shared memory", n, smem);
        return SPB_ERR_INVALID;
    }
    int blocks = sms < kNoAllocMaxBlocks ? sms : kNoAllocMaxBlocks;
    unsigned long long max_blocks = (pb.units + threads - 1) / threads;
    if ((unsigned long long)blocks > max_blocks) blocks = (int)max_blocks;
    if (blocks < 1) blocks = 1;
    pb.grid = blocks;
    pb.threads = threads;

    size_t in_off = 0;
    const size_t need = plan_layout(&pb, nullptr, &in_off);
    if (need > kNoAllocScratchBytes) {
        spb_set_error("spb_perm_dense_f64_noalloc: n=%d needs %zu B of working memory, more "
                      "than the fixed %zu B", n, need, kNoAllocScratchBytes);
        return SPB_ERR_INVALID;
    }
    plan_layout(&pb, static_cast<char*>(g_scratch_ptr[dev]), &in_off);

    // setup_kernel zeroes the ticket the walk's grid reduction counts on.
    int st0 = launch_setup(pb, d_a, s);
    if (st0 != SPB_OK) return st0;
    int st = launch_walk(pb, blocks, threads, smem, s);
    if (st != SPB_OK) return st;
    noalloc_finalize<<<1, 32, 0, s>>>(pb, d_out);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}
