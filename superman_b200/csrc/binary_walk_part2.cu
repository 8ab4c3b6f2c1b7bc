// walk_binary<N, L> instantiations (L=10, L=6).
#include "binary_launch.cuh"

namespace spb {
namespace binary {

template int launch_bin_n<34, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<35, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<36, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<37, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<38, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<39, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<40, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<41, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<42, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<43, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<44, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<45, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<46, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<47, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<48, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<49, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<50, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<51, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<52, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<53, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<54, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<55, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<56, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<57, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<58, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<59, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<60, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<61, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<62, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<63, 6>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<46, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<47, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<48, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<49, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<50, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<51, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<52, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<53, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<54, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<55, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<56, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<57, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<58, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<59, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<60, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<61, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<62, 10>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_bin_n<63, 10>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace binary
}  // namespace spb
