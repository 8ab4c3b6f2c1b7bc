// Per-(n, limbs) launch helper for walk_binary, instantiated in
// binary_walk_part*.cu and dispatched in binary_dispatch.cu.
#pragma once

#include <mutex>

#include "binary_impl.cuh"

namespace spb {
namespace binary {

// With per_sm set, launches nothing and stores how many CTAs of `threads`
// threads and `smem` bytes fit on one SM.
template <int N, int L>
int launch_bin_n(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s, int* per_sm)
{
    static std::once_flag once[64];
    static cudaError_t attr_err[64];
    int dev = 0;
    SPB_CUDA_TRY(cudaGetDevice(&dev));
    std::call_once(once[dev & 63], [&] {
        int optin = 0;
        cudaFuncAttributes fa{};
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        attr_err[dev & 63] = cudaFuncGetAttributes(&fa, walk_binary<N, L>);
        if (attr_err[dev & 63] == cudaSuccess)
            attr_err[dev & 63] = cudaFuncSetAttribute(walk_binary<N, L>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      optin - (int)fa.sharedSizeBytes);
    });
    SPB_CUDA_TRY(attr_err[dev & 63]);
    if (per_sm) {
        SPB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, walk_binary<N, L>, threads, smem));
        return SPB_OK;
    }
    walk_binary<N, L><<<blocks, threads, smem, s>>>(pb);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

}  // namespace binary
}  // namespace spb
