// walk_complex<N> instantiations for n = 21..30.
#include "dense_launch.cuh"

namespace spb {
namespace dense {

SPB_DEFINE_LAUNCH(launch_complex_n, walk_complex)

template int launch_complex_n<21>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<22>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<23>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<24>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<25>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<26>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<27>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<28>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<29>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<30>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
