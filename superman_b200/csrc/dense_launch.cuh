// Per-n launch helpers for the dense walk kernels.  Instantiated in the
// dense_walk_{real,complex}_part*.cu units (split for parallel compilation)
// and dispatched on n in dense_dispatch.cu.
#pragma once

#include <mutex>

#include "dense_impl.cuh"

namespace spb {
namespace dense {

template <int N>
int launch_real_n(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s);
template <int N>
int launch_complex_n(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s);

#define SPB_DEFINE_LAUNCH(NAME, KERNEL)                                                         \
    template <int N>                                                                            \
    int NAME(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s)           \
    {                                                                                           \
        static std::once_flag once[64];                                                         \
        static cudaError_t attr_err[64];                                                        \
        int dev = 0;                                                                            \
        SPB_CUDA_TRY(cudaGetDevice(&dev));                                                      \
        std::call_once(once[dev & 63], [&] {                                                    \
            int optin = 0;                                                                      \
            cudaFuncAttributes fa{};                                                            \
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);       \
            attr_err[dev & 63] = cudaFuncGetAttributes(&fa, KERNEL<N>);                         \
            if (attr_err[dev & 63] == cudaSuccess)                                              \
                attr_err[dev & 63] = cudaFuncSetAttribute(                                      \
                    KERNEL<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,                     \
                    optin - (int)fa.sharedSizeBytes);                                           \
        });                                                                                     \
        SPB_CUDA_TRY(attr_err[dev & 63]);                                                       \
        if (blocks <= 0) return SPB_OK; /* prepare only: kernel loaded, attributes set */       \
        KERNEL<N><<<blocks, threads, smem, s>>>(pb);                                            \
        SPB_CUDA_TRY(cudaGetLastError());                                                       \
        return SPB_OK;                                                                          \
    }

}  // namespace dense
}  // namespace spb
