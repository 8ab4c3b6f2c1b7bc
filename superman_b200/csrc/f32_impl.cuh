// FP32-product walk (precision SPB_PREC_FP32), real and complex, n <= 40.
//
// The same formulation as the FP64 walks (dense_impl.cuh): low columns from a
// subset-sum table, high columns walked in Gray order as units with
// double-double unit bases (hi in registers, lo in shared memory).  What
// changes is the arithmetic of a term.  The unit base is rounded to float once
// per unit, the table is read as floats (setup_kernel writes de32), and a
// term's row values x_r = xf_r + DE32[d][r] and their product are FP32
// operations, twice the FP64 pipe's rate on B200.  Each group of terms is
// combined in FP64, and units and the grid total are summed in double-double
// as in the FP64 walk.  A term's relative error is of order n * 2^-24, so the
// result's is of order kappa * n * 2^-24, with kappa = sqrt(sum t^2) / |sum t|.
// That suits inputs whose kappa is small, e.g. Haar-random complex blocks.
// The walk also sums every term's square (|t|^2 for complex) into
// pb.rb->err (zeroed by setup_kernel), from which the host estimates the
// result's relative error and refuses the result when it exceeds the
// caller's bound.
#pragma once

#include "dense_impl.cuh"

namespace spb {
namespace dense {

template <int N, int C>
struct F32Cfg {
    // the table's grouping is the one setup_kernel lays out (group_size)
    static constexpr int G = C == 1 ? RealCfg<N>::G : ComplexCfg<N>::G;
    static constexpr int kMaxThreads = (C == 1 && N <= 32) ? 512 : 256;
};

__host__ __device__ inline size_t f32_smem_bytes(int n, int c, int w, int threads)
{
    const size_t terms = (size_t)1 << w, ntp = n - 1 - w > 0 ? n - 1 - w : 0;
    return sizeof(float) * c * terms * n + sizeof(double) * (c * ntp * n + (size_t)c * n * threads);
}

template <int N, int C>
__global__ void __launch_bounds__(F32Cfg<N, C>::kMaxThreads, 1) walk_f32(Problem pb)
{
    constexpr int G = F32Cfg<N, C>::G;
    extern __shared__ __align__(16) double smem[];
    const int w = pb.w, terms = 1 << w, nq = terms / G, ntop = N - 1 - w, ntp = ntop > 0 ? ntop : 0;
    const int tid = threadIdx.x, bd = blockDim.x;
    float* s_de = reinterpret_cast<float*>(smem);  // [C][nq][N][G]
    // C*terms*N floats is a multiple of 4 (terms >= 4), so the doubles stay aligned
    double* s_mt = smem + (size_t)C * terms * N / 2;  // [C][ntop][N]
    double* s_lo = s_mt + C * ntp * N;                // [C][N][bd]
    for (int i = tid; i < C * terms * N; i += bd) s_de[i] = pb.de32[i];
    for (int i = tid; i < C * ntp * N; i += bd) s_mt[i] = pb.mt[i];
    __syncthreads();

    const unsigned long long T = (unsigned long long)gridDim.x * bd;
    const unsigned long long t = (unsigned long long)blockIdx.x * bd + tid;
    unsigned long long u0, u1;
    balanced_range(pb.units, T, t, &u0, &u1);
    dd tot[C];
#pragma unroll
    for (int c = 0; c < C; ++c) tot[c] = {0.0, 0.0};
    double s2 = 0.0;  // sum of squared terms (the error estimate's input)
    if (u0 < u1) {
        double xh[C][N];
        const unsigned long long g0 = gray_of(u0);
        // R rows of every part (four add chains) at a time, the same
        // operations per row.
        constexpr int R = 4 / C;
#pragma unroll
        for (int r0 = 0; r0 < N; r0 += R) {
            dd x[C][R];
#pragma unroll
            for (int c = 0; c < C; ++c)
#pragma unroll
                for (int k = 0; k < R; ++k)
                    if (r0 + k < N) x[c][k] = dd{pb.x0_hi[c * N + r0 + k], pb.x0_lo[c * N + r0 + k]};
            for (int j = 0; j < ntop; ++j)
                if ((g0 >> j) & 1ull) {
#pragma unroll
                    for (int c = 0; c < C; ++c)
#pragma unroll
                        for (int k = 0; k < R; ++k)
                            if (r0 + k < N) x[c][k] = dd_add_d(x[c][k], s_mt[(c * ntp + j) * N + r0 + k]);
                }
#pragma unroll
            for (int c = 0; c < C; ++c)
#pragma unroll
                for (int k = 0; k < R; ++k)
                    if (r0 + k < N) {
                        xh[c][r0 + k] = x[c][k].hi;
                        s_lo[(c * N + r0 + k) * bd + tid] = x[c][k].lo;
                    }
        }
        unsigned long long u = u0;
        while (true) {
            float xf[C][N];
#pragma unroll
            for (int c = 0; c < C; ++c)
#pragma unroll
                for (int r = 0; r < N; ++r) xf[c][r] = __double2float_rn(xh[c][r]);
            double acc[C];
#pragma unroll
            for (int c = 0; c < C; ++c) acc[c] = 0.0;
#pragma unroll 1
            for (int q = 0; q < nq; ++q) {
                double gsum[C];
                if constexpr (C == 1) {
                    const float* de = s_de + q * (N * G);
                    float p[G];
#pragma unroll
                    for (int i = 0; i < G; ++i) p[i] = __fadd_rn(xf[0][0], de[i]);
#pragma unroll
                    for (int r = 1; r < N; ++r) {
                        if constexpr (G == 4) {
                            const float4 v = reinterpret_cast<const float4*>(de + r * 4)[0];
                            p[0] = __fmul_rn(p[0], __fadd_rn(xf[0][r], v.x));
                            p[1] = __fmul_rn(p[1], __fadd_rn(xf[0][r], v.y));
                            p[2] = __fmul_rn(p[2], __fadd_rn(xf[0][r], v.z));
                            p[3] = __fmul_rn(p[3], __fadd_rn(xf[0][r], v.w));
                        } else {
#pragma unroll
                            for (int i = 0; i < G; ++i) p[i] = __fmul_rn(p[i], __fadd_rn(xf[0][r], de[r * G + i]));
                        }
                    }
                    if constexpr (G == 4)
                        gsum[0] = ((double)p[0] - (double)p[1]) - ((double)p[2] - (double)p[3]);  // + - - +
                    else if constexpr (G == 2)
                        gsum[0] = (double)p[0] - (double)p[1];
                    else
                        gsum[0] = (double)p[0];
#pragma unroll
                    for (int i = 0; i < G; ++i) s2 = __fma_rn((double)p[i], (double)p[i], s2);
                } else {
                    const float* dr = s_de + q * (N * G);
                    const float* di = s_de + terms * N + q * (N * G);
                    float pr[G], pi[G];
#pragma unroll
                    for (int i = 0; i < G; ++i) {
                        pr[i] = __fadd_rn(xf[0][0], dr[i]);
                        pi[i] = __fadd_rn(xf[1][0], di[i]);
                    }
#pragma unroll
                    for (int r = 1; r < N; ++r) {
                        float vr[G], vi[G];
                        if constexpr (G == 4) {  // two 16-byte loads per row
                            const float4 a = reinterpret_cast<const float4*>(dr + r * 4)[0];
                            const float4 b = reinterpret_cast<const float4*>(di + r * 4)[0];
                            vr[0] = a.x; vr[1] = a.y; vr[2] = a.z; vr[3] = a.w;
                            vi[0] = b.x; vi[1] = b.y; vi[2] = b.z; vi[3] = b.w;
                        } else {
#pragma unroll
                            for (int i = 0; i < G; ++i) { vr[i] = dr[r * G + i]; vi[i] = di[r * G + i]; }
                        }
#pragma unroll
                        for (int i = 0; i < G; ++i) {
                            const float yr = __fadd_rn(xf[0][r], vr[i]);
                            const float yi = __fadd_rn(xf[1][r], vi[i]);
                            const float t1 = __fmul_rn(pi[i], yi);
                            const float t2 = __fmul_rn(pi[i], yr);
                            const float nr = __fmaf_rn(pr[i], yr, -t1);
                            const float ni = __fmaf_rn(pr[i], yi, t2);
                            pr[i] = nr;
                            pi[i] = ni;
                        }
                    }
                    if constexpr (G == 4) {
                        gsum[0] = ((double)pr[0] - (double)pr[1]) - ((double)pr[2] - (double)pr[3]);
                        gsum[1] = ((double)pi[0] - (double)pi[1]) - ((double)pi[2] - (double)pi[3]);
                    } else if constexpr (G == 2) {
                        gsum[0] = (double)pr[0] - (double)pr[1];
                        gsum[1] = (double)pi[0] - (double)pi[1];
                    } else {
                        gsum[0] = (double)pr[0];
                        gsum[1] = (double)pi[0];
                    }
#pragma unroll
                    for (int i = 0; i < G; ++i)
                        s2 = __fma_rn((double)pi[i], (double)pi[i], __fma_rn((double)pr[i], (double)pr[i], s2));
                }
#pragma unroll
                for (int c = 0; c < C; ++c) acc[c] = (__popc(q) & 1) ? acc[c] - gsum[c] : acc[c] + gsum[c];
            }
#pragma unroll
            for (int c = 0; c < C; ++c) tot[c] = dd_add_d(tot[c], (u & 1ull) ? -acc[c] : acc[c]);
            if (++u >= u1) break;
            const int j = __ffsll((long long)u) - 1;
            const bool add = (gray_of(u) >> j) & 1ull;
#pragma unroll
            for (int c = 0; c < C; ++c)
#pragma unroll
                for (int r = 0; r < N; ++r) {
                    const double m = add ? s_mt[(c * ntp + j) * N + r] : -s_mt[(c * ntp + j) * N + r];
                    const dd s = two_sum(xh[c][r], m);
                    const dd z = fast_two_sum(s.hi, add_rn(s.lo, s_lo[(c * N + r) * bd + tid]));
                    xh[c][r] = z.hi;
                    s_lo[(c * N + r) * bd + tid] = z.lo;
                }
        }
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, m);
    if ((tid & 31) == 0) atomicAdd(&pb.rb->err, s2);
    grid_reduce<C>(tot, pb);
}

}  // namespace dense
}  // namespace spb

#include <mutex>
#include <set>
#include <utility>

namespace spb {
namespace dense {

// Launches walk_f32<N, C>, first raising its dynamic shared-memory limit to
// the opt-in maximum (once per device).
template <int N, int C>
int launch_f32_n(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s)
{
    static std::mutex mu;
    static std::set<int> done;
    int dev = 0;
    SPB_CUDA_TRY(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!done.count(dev)) {
            int optin = 0;
            cudaFuncAttributes fa{};
            SPB_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
            SPB_CUDA_TRY(cudaFuncGetAttributes(&fa, walk_f32<N, C>));
            SPB_CUDA_TRY(cudaFuncSetAttribute(walk_f32<N, C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              optin - (int)fa.sharedSizeBytes));
            done.insert(dev);
        }
    }
    walk_f32<N, C><<<blocks, threads, smem, s>>>(pb);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

}  // namespace dense
}  // namespace spb
