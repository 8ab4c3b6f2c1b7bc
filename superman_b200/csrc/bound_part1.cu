// bound_walk<N, C> instantiations for n = 32..63.
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

template int launch_bound_n<32>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<33>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<34>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<35>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<36>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<37>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<38>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<39>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<40>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<41>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<42>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<43>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<44>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<45>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<46>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<47>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<48>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<49>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<50>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<51>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<52>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<53>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<54>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<55>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<56>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<57>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<58>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<59>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<60>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<61>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<62>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bound_n<63>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
