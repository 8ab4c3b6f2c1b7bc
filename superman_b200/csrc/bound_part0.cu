// bound_walk<N, C> instantiations for n = 1..31.
#include "bound_impl.cuh"
#include "dense_launch.cuh"

namespace spb {
namespace dense {

template <int N>
int launch_bound_n(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s)
{
    if (pb.comps == 1) {
        SPB_CUDA_TRY(cudaFuncSetAttribute(bound_walk<N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        bound_walk<N, 1><<<blocks, threads, smem, s>>>(pb);
    } else {
        SPB_CUDA_TRY(cudaFuncSetAttribute(bound_walk<N, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        bound_walk<N, 2><<<blocks, threads, smem, s>>>(pb);
    }
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

template int launch_bound_n<1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<3>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<4>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<5>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<7>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<8>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<9>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<11>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<12>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<13>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<14>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<15>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<16>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<17>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<18>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<19>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<20>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<21>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<22>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<23>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<24>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<25>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<26>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<27>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<28>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<29>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<30>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<31>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
