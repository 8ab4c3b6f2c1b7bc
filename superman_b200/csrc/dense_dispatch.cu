// Run-time dispatch of the dense walk kernels on n.
#include "dense_launch.cuh"

namespace spb {
namespace dense {

int launch_walk_real(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s)
{
    switch (pb.n) {
#define SPB_CASE(N) \
    case N: return launch_real_n<N>(pb, blocks, threads, smem, s);
        SPB_FOR_EACH_N(SPB_CASE)
#undef SPB_CASE
    default:
        spb_set_error("dense walk: n=%d outside 1..%d", pb.n, kMaxN);
        return SPB_ERR_INVALID;
    }
}

int launch_walk_complex(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s)
{
    switch (pb.n) {
#define SPB_CASE(N) \
    case N: return launch_complex_n<N>(pb, blocks, threads, smem, s);
        SPB_FOR_EACH_N(SPB_CASE)
#undef SPB_CASE
    default:
        spb_set_error("dense walk: n=%d outside 1..%d", pb.n, kMaxN);
        return SPB_ERR_INVALID;
    }
}

int prepare_walk_real(int n)
{
    Problem pb{};
    pb.n = n;
    pb.na = n;
    pb.comps = 1;
    return launch_walk_real(pb, 0, 0, 0, nullptr);  // blocks = 0: load and configure, no launch
}

int walk_max_threads(int n, int comps)
{
    return comps == 1 ? RealMaxThreads(n) : ComplexMaxThreads(n);
}

}  // namespace dense
}  // namespace spb
