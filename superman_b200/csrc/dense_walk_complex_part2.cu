// walk_complex<N> instantiations for n = 31..40.
#include "dense_launch.cuh"

namespace spb {
namespace dense {

SPB_DEFINE_LAUNCH(launch_complex_n, walk_complex)

template int launch_complex_n<31>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<32>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<33>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<34>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<35>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<36>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<37>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<38>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<39>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<40>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
