// walk_sparse<NA> instantiations for NA = 17..32 active rows.
#include "dense_launch.cuh"
#include "sparse_impl.cuh"

namespace spb {
namespace dense {

SPB_DEFINE_LAUNCH(launch_sparse_na, walk_sparse)

template int launch_sparse_na<17>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<18>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<19>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<20>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<21>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<22>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<23>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<24>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<25>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<26>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<27>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<28>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<29>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<30>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<31>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_sparse_na<32>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
