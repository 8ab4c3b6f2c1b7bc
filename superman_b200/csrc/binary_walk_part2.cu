// walk_binary<N, L> instantiations (L=5 n=22..42).
#include "binary_launch.cuh"

namespace spb {
namespace binary {

template int launch_bin_n<22, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<23, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<24, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<25, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<26, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<27, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<28, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<29, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<30, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<31, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<32, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<33, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<34, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<35, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<36, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<37, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<38, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<39, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<40, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<41, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<42, 5>(const Problem&, int, int, size_t, cudaStream_t, int*);

}  // namespace binary
}  // namespace spb
