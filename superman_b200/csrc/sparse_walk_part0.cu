// walk_sparse<NA> instantiations for NA = 1..16 active rows.
#include "dense_launch.cuh"
#include "sparse_impl.cuh"

namespace spb {
namespace dense {

SPB_DEFINE_LAUNCH(launch_sparse_na, walk_sparse)

template int launch_sparse_na<1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<3>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<4>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<5>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<7>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<8>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<9>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<11>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<12>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<13>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<14>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<15>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<16>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
