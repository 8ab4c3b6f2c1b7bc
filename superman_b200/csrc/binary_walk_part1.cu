// walk_binary<N, L> instantiations (L=4 n=34..63).
#include "binary_launch.cuh"

namespace spb {
namespace binary {

template int launch_bin_n<34, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<35, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<36, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<37, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<38, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<39, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<40, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<41, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<42, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<43, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<44, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<45, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<46, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<47, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<48, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<49, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<50, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<51, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<52, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<53, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<54, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<55, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<56, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<57, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<58, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<59, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<60, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<61, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<62, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<63, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);

}  // namespace binary
}  // namespace spb
