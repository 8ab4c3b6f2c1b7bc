// walk_binary<N, L> instantiations (L=10 n=38..63, L=12 n=56..63).
#include "binary_launch.cuh"

namespace spb {
namespace binary {

template int launch_bin_n<38, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<39, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<40, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<41, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<42, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<43, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<44, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<45, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<46, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<47, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<48, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<49, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<50, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<51, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<52, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<53, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<54, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<55, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<56, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<57, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<58, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<59, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<60, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<61, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<62, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<63, 10>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<56, 12>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<57, 12>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<58, 12>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<59, 12>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<60, 12>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<61, 12>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<62, 12>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<63, 12>(const Problem&, int, int, size_t, cudaStream_t, int*);

}  // namespace binary
}  // namespace spb
