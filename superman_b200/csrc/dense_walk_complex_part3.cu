// walk_complex<N> instantiations for n = 41..63.
#include "dense_launch.cuh"

namespace spb {
namespace dense {

SPB_DEFINE_LAUNCH(launch_complex_n, walk_complex)

template int launch_complex_n<41>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<42>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<43>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<44>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<45>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<46>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<47>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<48>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<49>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<50>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<51>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<52>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<53>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<54>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<55>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<56>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<57>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<58>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<59>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<60>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<61>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<62>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_complex_n<63>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
