// walk_real<N> instantiations for n = 41..63.
#include "dense_launch.cuh"

namespace spb {
namespace dense {

SPB_DEFINE_LAUNCH(launch_real_n, walk_real)

template int launch_real_n<41>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<42>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<43>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<44>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<45>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<46>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<47>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<48>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<49>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<50>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<51>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<52>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<53>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<54>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<55>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<56>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<57>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<58>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<59>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<60>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<61>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<62>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_real_n<63>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
