// walk_binary<N, L> instantiations (L=5 n=43..63).
#include "binary_launch.cuh"

namespace spb {
namespace binary {

template int launch_bin_n<43, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<44, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<45, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<46, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<47, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<48, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<49, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<50, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<51, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<52, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<53, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<54, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<55, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<56, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<57, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<58, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<59, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<60, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<61, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<62, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<63, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);

}  // namespace binary
}  // namespace spb
