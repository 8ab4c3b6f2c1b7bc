// Row-compacted walk for sparse real matrices (the B200 counterpart of the
// reference's sparse kernels, Algorithms/GPU/Sparse/SparseKernelDefinitions.cuh,
// and of its per-matrix generated kernels, Algorithms/GPU/CodeGeneration/).
//
// The host (sparse.cu) permutes rows and columns so that
//   * columns 0..w-1 are the w "low" columns whose row supports have the
//     smallest union, column n-1 is the Nijenhuis–Wilf last column;
//   * rows 0..NA-1 are the rows with a nonzero in some low column ("active"),
//     rows NA..n-1 have none ("inactive").
// Within a unit (fixed high-column subset) an inactive row's x_r = xtop_r does
// not depend on the low subset d, so its factor is common to all 2^w terms:
//   term_d = c * prod_{r < NA} (xtop_r + DE[d][r]),  c = prod_{r >= NA} xtop_r.
// A term costs 2*NA FP64 operations instead of 2n; c costs n-NA per unit.
// Active unit bases are double-double with hi in registers (as in the dense
// walk); inactive ones are double-double in shared memory and a Gray step
// touches only the nonzeros of the flipped high column among them.
//
// The FP64 arithmetic of a term is fixed: c = x_NA * x_{NA+1} * ... * x_{n-1}
// (left to right), then p = c * (xtop_0 + DE[d][0]), then the active rows in
// order.  refine_real (dense_refine.cu) replays exactly this when pb.na < pb.n.
#pragma once

#include "dense_impl.cuh"

namespace spb {
namespace dense {

// Highest active-row count with a compiled kernel.
constexpr int kMaxActive = 32;

template <int NA, bool STATS = false>
__device__ __forceinline__ double unit_sum_sparse(const double (&xa)[NA], double c,
                                                  const double* __restrict__ s_de, int nq,
                                                  double* s2 = nullptr)
{
    double acc = 0.0, sq[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
    for (int q = 0; q < nq; ++q) {
        const double* de = s_de + q * (NA * 4);
        double p[4];
        {
            double2 v0 = reinterpret_cast<const double2*>(de)[0];
            double2 v1 = reinterpret_cast<const double2*>(de)[1];
            p[0] = mul_rn(c, add_rn(xa[0], v0.x));
            p[1] = mul_rn(c, add_rn(xa[0], v0.y));
            p[2] = mul_rn(c, add_rn(xa[0], v1.x));
            p[3] = mul_rn(c, add_rn(xa[0], v1.y));
        }
#pragma unroll
        for (int r = 1; r < NA; ++r) {
            double2 a = reinterpret_cast<const double2*>(de + r * 4)[0];
            double2 b = reinterpret_cast<const double2*>(de + r * 4)[1];
            p[0] = mul_rn(p[0], add_rn(xa[r], a.x));
            p[1] = mul_rn(p[1], add_rn(xa[r], a.y));
            p[2] = mul_rn(p[2], add_rn(xa[r], b.x));
            p[3] = mul_rn(p[3], add_rn(xa[r], b.y));
        }
        const double gs = sub_rn(sub_rn(p[0], p[1]), sub_rn(p[2], p[3]));  // + - - +
        acc = (__popc(q) & 1) ? sub_rn(acc, gs) : add_rn(acc, gs);
        if constexpr (STATS) {
#pragma unroll
            for (int i = 0; i < 4; ++i) sq[i] = __fma_rn(p[i], p[i], sq[i]);
        }
    }
    if constexpr (STATS) *s2 = (sq[0] + sq[1]) + (sq[2] + sq[3]);
    return acc;
}

// Shared memory of walk_sparse: tables, per-thread unit bases, histogram.
__host__ __device__ inline size_t sparse_smem_bytes(int n, int na, int w, int threads)
{
    const size_t terms = (size_t)1 << w, ntop = n - 1 - w, ni = n - na;
    size_t b = sizeof(double) * (terms * na + ntop * na + ntop * ni + (size_t)(na + 2 * ni) * threads);
    b += kHistSmemBytes + sizeof(double) * 2 * na;
    b += ntop * ni + ntop;  // inactive row indices and counts (bytes)
    return (b + 15) / 16 * 16;
}

template <int NA>
__global__ void __launch_bounds__(512, 1) walk_sparse(Problem pb)
{
    extern __shared__ __align__(16) double smem[];
    const int n = pb.n, w = pb.w, terms = 1 << w, nq = terms / 4;
    const int ntop = n - 1 - w, ni = n - NA;
    const int tid = threadIdx.x, bd = blockDim.x;
    double* s_de = smem;                   // [nq][NA][4] active rows of DE
    double2* s_bnd = reinterpret_cast<double2*>(s_de + terms * NA);  // [NA] DE range (min, max)
    double* s_ma = reinterpret_cast<double*>(s_bnd + NA);  // [ntop][NA] active part of the high columns
    double* s_iv = s_ma + ntop * NA;       // [ntop][ni] inactive nonzeros, compacted per column
    double* s_lo = s_iv + ntop * ni;       // [NA][bd] active lo words
    double* s_ih = s_lo + NA * bd;         // [ni][bd] inactive hi words
    double* s_il = s_ih + ni * bd;         // [ni][bd] inactive lo words
    float* s_hist = reinterpret_cast<float*>(s_il + ni * bd);  // mode 1
    unsigned* s_cnt = reinterpret_cast<unsigned*>(s_hist + kHistBins);
    unsigned char* s_ir = reinterpret_cast<unsigned char*>(s_cnt + kHistBins);  // [ntop][ni]
    unsigned char* s_ic = s_ir + ntop * ni;                                   // [ntop]

    for (int i = tid; i < terms * NA; i += bd) {
        const int q = i / (NA * 4), rem = i % (NA * 4);
        s_de[i] = pb.de_hi[(size_t)q * n * 4 + rem];  // rows r < NA keep their [r][4] slots
    }
    for (int i = tid; i < ntop * NA; i += bd) s_ma[i] = pb.mt[(size_t)(i / NA) * n + (i % NA)];
    for (int j = tid; j < ntop; j += bd) {
        int cnt = 0;
        for (int k = 0; k < ni; ++k) {
            const double v = pb.mt[(size_t)j * n + NA + k];
            if (v != 0.0) {
                s_iv[j * ni + cnt] = v;
                s_ir[j * ni + cnt] = (unsigned char)k;
                ++cnt;
            }
        }
        s_ic[j] = (unsigned char)cnt;
    }
    const int mode = pb.mode;
    if (mode != 0)
        for (int r = tid; r < NA; r += bd) s_bnd[r] = make_double2(pb.bnd[r], pb.bnd[n + r]);
    if (mode == 1)
        for (int i = tid; i < kHistBins; i += bd) { s_hist[i] = 0.0f; s_cnt[i] = 0u; }
    __syncthreads();

    const unsigned long long T = (unsigned long long)gridDim.x * bd;
    const unsigned long long t = (unsigned long long)blockIdx.x * bd + tid;
    unsigned long long u0, u1;
    balanced_range(pb.units, T, t, &u0, &u1);
    if (mode == 2 && (int)pb.tmax[t] < pb.thr_bin) u1 = u0;
    dd tot[1] = {{0.0, 0.0}};
    HistCache hc;
    const int lbin = mode == 1 ? __ldcg(pb.list_bin) : 0;
    int bmax = 0;
    if (u0 < u1) {
        double xa[NA];
        const unsigned long long g0 = gray_of(u0);
        // First unit base: x0 plus the selected high columns in index order,
        // zeros included (the same operations as the refinement's rebuild).
        // Four rows at a time: independent add chains, the same operations per row.
#pragma unroll
        for (int r0 = 0; r0 < NA; r0 += 4) {
            dd x[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (r0 + k < NA) x[k] = dd{pb.x0_hi[r0 + k], pb.x0_lo[r0 + k]};
            for (int j = 0; j < ntop; ++j)
                if ((g0 >> j) & 1ull) {
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (r0 + k < NA) x[k] = dd_add_d(x[k], s_ma[j * NA + r0 + k]);
                }
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (r0 + k < NA) {
                    xa[r0 + k] = x[k].hi;
                    s_lo[(r0 + k) * bd + tid] = x[k].lo;
                }
        }
        for (int k = 0; k < ni; ++k) {
            dd x = {pb.x0_hi[NA + k], pb.x0_lo[NA + k]};
            for (int j = 0; j < ntop; ++j)
                if ((g0 >> j) & 1ull) x = dd_add_d(x, pb.mt[(size_t)j * n + NA + k]);
            s_ih[k * bd + tid] = x.hi;
            s_il[k * bd + tid] = x.lo;
        }
        unsigned long long u = u0;
        while (true) {
            double c = s_ih[tid];
            for (int k = 1; k < ni; ++k) c = mul_rn(c, s_ih[k * bd + tid]);
            int b = 0;
            if (mode != 0) {
                double ub = fabs(c);
#pragma unroll
                for (int r = 0; r < NA; ++r) {
                    const double2 bb = s_bnd[r];
                    ub = mul_rn(ub, fmax(fabs(add_rn(xa[r], bb.x)), fabs(add_rn(xa[r], bb.y))));
                }
                b = hist_bin(ub);
                bmax = b > bmax ? b : bmax;
                if (mode == 2 && b >= pb.thr_bin) {
                    unsigned long long k = atomicAdd(pb.list_n, 1ull);
                    if (k < pb.list_cap) {
                        pb.list_u[k] = u;
                        double* dst = pb.list_x + k * (2 * (size_t)n);
#pragma unroll
                        for (int r = 0; r < NA; ++r) { dst[r] = xa[r]; dst[n + r] = s_lo[r * bd + tid]; }
                        for (int i = 0; i < ni; ++i) {
                            dst[NA + i] = s_ih[i * bd + tid];
                            dst[n + NA + i] = s_il[i * bd + tid];
                        }
                    }
                }
            }
            if (mode == 0) {
                const double us = unit_sum_sparse<NA>(xa, c, s_de, nq);
                tot[0] = dd_add_d(tot[0], (u & 1ull) ? -us : us);
            } else if (mode == 1) {
                double sq;
                const double us = unit_sum_sparse<NA, true>(xa, c, s_de, nq, &sq);
                tot[0] = dd_add_d(tot[0], (u & 1ull) ? -us : us);
                hc.add(b, sq, s_hist, s_cnt);
                raw_list_add(pb, lbin, u, b);
            }
            if (++u >= u1) break;
            const int j = __ffsll((long long)u) - 1;
            const bool add = (gray_of(u) >> j) & 1ull;
            const double* col = s_ma + j * NA;
#pragma unroll
            for (int r = 0; r < NA; ++r) {
                const double m = add ? col[r] : -col[r];
                dd s = two_sum(xa[r], m);
                dd z = fast_two_sum(s.hi, add_rn(s.lo, s_lo[r * bd + tid]));
                xa[r] = z.hi;
                s_lo[r * bd + tid] = z.lo;
            }
            // Adding a zero leaves a normalised double-double unchanged, so only
            // the column's inactive nonzeros are applied.
            const int cnt = s_ic[j];
            for (int k = 0; k < cnt; ++k) {
                const int i = s_ir[j * ni + k];
                const double m = add ? s_iv[j * ni + k] : -s_iv[j * ni + k];
                dd s = two_sum(s_ih[i * bd + tid], m);
                dd z = fast_two_sum(s.hi, add_rn(s.lo, s_il[i * bd + tid]));
                s_ih[i * bd + tid] = z.hi;
                s_il[i * bd + tid] = z.lo;
            }
        }
    }
    if (mode == 1) {
        pb.tmax[t] = (unsigned short)bmax;
        hc.flush(s_hist, s_cnt);
        __syncthreads();
        flush_hist(s_hist, s_cnt, pb);
    }
    if (mode != 2) grid_reduce<1>(tot, pb);
}

}  // namespace dense
}  // namespace spb
