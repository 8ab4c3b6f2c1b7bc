// walk_complex<N> instantiations for n = 1..20.
#include "dense_launch.cuh"

namespace spb {
namespace dense {

SPB_DEFINE_LAUNCH(launch_complex_n, walk_complex)

template int launch_complex_n<1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<3>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<4>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<5>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<7>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<8>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<9>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<11>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<12>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<13>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<14>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<15>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<16>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<17>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<18>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<19>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<20>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
