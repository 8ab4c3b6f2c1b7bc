// walk_f32<N, 1> (real, FP32 products) instantiations for n = 3..40.
#include "f32_impl.cuh"

namespace spb {
namespace dense {

template int launch_f32_n<3, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<4, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<5, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<6, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<7, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<8, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<9, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<10, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<11, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<12, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<13, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<14, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<15, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<16, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<17, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<18, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<19, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<20, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<21, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<22, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<23, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<24, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<25, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<26, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<27, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<28, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<29, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<30, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<31, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<32, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<33, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<34, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<35, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<36, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<37, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<38, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<39, 1>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<40, 1>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
