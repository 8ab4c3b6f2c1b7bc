// walk_f32<N, 2> (complex, FP32 products) instantiations for n = 3..40.
#include "f32_impl.cuh"

namespace spb {
namespace dense {

template int launch_f32_n<3, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<4, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<5, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<6, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<7, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<8, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<9, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<10, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<11, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<12, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<13, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<14, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<15, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<16, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<17, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<18, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<19, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<20, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<21, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<22, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<23, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<24, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<25, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<26, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<27, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<28, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<29, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<30, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<31, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<32, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<33, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<34, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<35, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<36, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<37, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<38, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<39, 2>(const Problem&, int, int, size_t, cudaStream_t);
template int launch_f32_n<40, 2>(const Problem&, int, int, size_t, cudaStream_t);

}  // namespace dense
}  // namespace spb
