// walk_binary<N, L> instantiations (L=4 n=3..33).
#include "binary_launch.cuh"

namespace spb {
namespace binary {

template int launch_bin_n<3, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<4, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<5, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<6, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<7, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<8, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<9, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<10, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<11, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<12, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<13, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<14, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<15, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<16, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<17, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<18, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<19, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<20, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<21, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<22, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<23, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<24, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<25, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<26, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<27, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<28, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<29, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<30, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<31, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<32, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);
template int launch_bin_n<33, 4>(const Problem&, int, int, size_t, cudaStream_t, int*);

}  // namespace binary
}  // namespace spb
