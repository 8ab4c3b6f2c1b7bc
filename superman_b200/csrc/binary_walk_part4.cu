// walk_binary<N, L> instantiations (L=6 n=28..45).
#include "binary_launch.cuh"

namespace spb {
namespace binary {

template int launch_bin_n<28, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<29, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<30, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<31, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<32, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<33, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<34, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<35, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<36, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<37, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<38, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<39, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<40, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<41, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<42, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<43, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<44, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<45, 6>(const Problem&, int, int, size_t, cudaStream_t, int*);

}  // namespace binary
}  // namespace spb
