// walk_binary<N, L> instantiations (L=6 n=46..63).
#include "binary_launch.cuh"

namespace spb {
namespace binary {

template int launch_bin_n<46, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<47, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<48, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<49, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<50, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<51, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<52, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<53, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<54, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<55, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<56, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<57, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<58, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<59, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<60, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<61, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<62, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<63, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);

}  // namespace binary
}  // namespace spb
