// walk_real<N> instantiations for n = 1..20.
#include "dense_launch.cuh"

namespace spb {
namespace dense {

SPB_DEFINE_LAUNCH(launch_real_n, walk_real)

template int launch_real_n<1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<3>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<4>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<5>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<7>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<8>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<9>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<11>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<12>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<13>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<14>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<15>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<16>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<17>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<18>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<19>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<20>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
