// Double-double re-evaluation of the dominant units (precision SPB_PREC_DD).
//
// Ryser's alternating sum is dominated, for many inputs, by a small set of
// very large terms (for positive matrices: subsets near the empty and the
// full set).  Their FP64 rounding errors, not the many small terms, set the
// final error.  The walk (mode 1) bins every unit by an upper bound U_u of its
// terms and accumulates the unit's actual sum of squared terms in that bin;
// the host picks the bin from which the remaining units' rounding error fits
// the tolerance.  The units at or above it come from the walk's own list
// (every unit at or above a bin chosen beforehand by bound_walk, when that
// bin is low enough), else from a parallel scan (scan_parallel), and only if
// either count disagrees with the histogram from a replay scan (walk mode 2,
// same launch shape, so the unit bases are bit-identical) that lists them
// with their double-double base vectors.  This kernel then re-evaluates each
// listed unit, one warp per unit:
//   * the FP64 unit sum exactly as the walk computed it (same operations in
//     the same order, so the same bits), spread over the lanes by group;
//   * the double-double unit sum (x_r = xtop_r + DE[d][r] in double-double,
//     double-double products and sum);
// and accumulates sign_u * (dd_sum - fp64_sum) into pb.result.  Adding that
// correction to the walk's total replaces the dominant units' FP64 values by
// their double-double values.
#include "bound_impl.cuh"
#include "dense_impl.cuh"

namespace spb {
namespace dense {
namespace {

// One group of G terms, bitwise identical to unit_sum_real<N,G>'s group
// (na == n) or to unit_sum_sparse<NA>'s (na < n: the inactive rows' product
// first, then the na active rows; see sparse_impl.cuh).
__device__ __forceinline__ double group_sum_real_rt(const double* xh, const double* de, int n, int na, int G)
{
    double p0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
    p0 = add_rn(xh[0], de[0]);
    if (G >= 2) p1 = add_rn(xh[0], de[1]);
    if (G == 4) {
        p2 = add_rn(xh[0], de[2]);
        p3 = add_rn(xh[0], de[3]);
    }
    if (na < n) {
        double c = xh[na];
        for (int r = na + 1; r < n; ++r) c = mul_rn(c, xh[r]);
        p0 = mul_rn(c, p0);
        p1 = mul_rn(c, p1);
        p2 = mul_rn(c, p2);
        p3 = mul_rn(c, p3);
    }
    for (int r = 1; r < na; ++r) {
        const double x = xh[r];
        p0 = mul_rn(p0, add_rn(x, de[r * G + 0]));
        if (G >= 2) p1 = mul_rn(p1, add_rn(x, de[r * G + 1]));
        if (G == 4) {
            p2 = mul_rn(p2, add_rn(x, de[r * G + 2]));
            p3 = mul_rn(p3, add_rn(x, de[r * G + 3]));
        }
    }
    if (G == 4) return sub_rn(sub_rn(p0, p1), sub_rn(p2, p3));
    if (G == 2) return sub_rn(p0, p1);
    return p0;
}

// One group of G (<= 4) complex terms, bitwise identical to unit_sum_complex<N,G>.
__device__ __forceinline__ void group_sum_complex_rt(const double* xr, const double* xi,
                                                     const double* dr, const double* di, int n,
                                                     int G, double& gr, double& gi)
{
    double pr[4] = {0.0, 0.0, 0.0, 0.0}, pi[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < G; ++i) {
        pr[i] = add_rn(xr[0], dr[i]);
        pi[i] = add_rn(xi[0], di[i]);
    }
    for (int r = 1; r < n; ++r) {
        for (int i = 0; i < G; ++i) {
            double yr = add_rn(xr[r], dr[r * G + i]);
            double yi = add_rn(xi[r], di[r * G + i]);
            double t1 = mul_rn(pi[i], yi);
            double t2 = mul_rn(pi[i], yr);
            double nr = __fma_rn(pr[i], yr, -t1);
            double ni = __fma_rn(pr[i], yi, t2);
            pr[i] = nr;
            pi[i] = ni;
        }
    }
    if (G == 4) {
        gr = sub_rn(sub_rn(pr[0], pr[1]), sub_rn(pr[2], pr[3]));
        gi = sub_rn(sub_rn(pi[0], pi[1]), sub_rn(pi[2], pi[3]));
    } else if (G == 2) {
        gr = sub_rn(pr[0], pr[1]);
        gi = sub_rn(pi[0], pi[1]);
    } else {
        gr = pr[0];
        gi = pi[0];
    }
}

// Unit base of unit u (component `part`) rebuilt from scratch in
// double-double the way the walk builds a thread's first unit (x0 plus the
// selected high columns in index order); lanes take rows.
__device__ __forceinline__ void unit_base(const Problem& pb, unsigned long long u, int part, int lane, double* hi,
                                          double* lo)
{
    const int n = pb.n, ntop = n - 1 - pb.w;
    const unsigned long long g = gray_of(u);
    const double* mt = pb.mt + (size_t)part * (ntop > 0 ? ntop : 0) * n;
    for (int r = lane; r < n; r += 32) {
        dd x = {pb.x0_hi[part * n + r], pb.x0_lo[part * n + r]};
        for (int j = 0; j < ntop; ++j)
            if ((g >> j) & 1ull) x = dd_add_d(x, mt[j * n + r]);
        hi[r] = x.hi;
        lo[r] = x.lo;
    }
}

// The walk's unit bound (dense_impl.cuh walk_real/walk_complex, and
// sparse_impl.cuh walk_sparse when pb.na < pb.n) from the hi words of a unit
// base (xh: [comps][n]): the same operations in the same order.
__device__ double unit_bound_rt(const Problem& pb, const double* xh)
{
    const int n = pb.n, na = pb.na;
    double ub = 1.0;
    if (pb.comps == 2) {
        for (int r = 0; r < n; ++r) {
            const double xr = xh[r], xi = xh[kMaxN + r];
            ub = mul_rn(ub, add_rn(__dsqrt_rn(__fma_rn(xr, xr, mul_rn(xi, xi))), pb.bnd[r]));
        }
        return ub;
    }
    if (na < n) {
        double c = xh[na];
        for (int r = na + 1; r < n; ++r) c = mul_rn(c, xh[r]);
        ub = fabs(c);
    }
    for (int r = 0; r < na; ++r)
        ub = mul_rn(ub, fmax(fabs(add_rn(xh[r], pb.bnd[r])), fabs(add_rn(xh[r], pb.bnd[n + r]))));
    return ub;
}

// Parallel listing of the units whose bin >= thr_bin.  The walk's threads
// whose highest bin reaches it (tmax) are visited one per warp; each lane
// takes a contiguous part of that thread's units, builds the first unit base
// from scratch in double-double and steps through the Gray order with the
// walk's own base update, evaluating the walk's bound per unit.  Lists unit
// indices only (the refine kernel rebuilds the bases).  A lane's bases start
// from a rebuild rather than from the walk's thread start, so a hi word could
// in principle differ from the walk's (a row value within ~2^-100 of a
// rounding midpoint); if that ever moved a unit across the threshold the
// count check fails and the caller falls back to the replay scan.
__global__ void __launch_bounds__(128) scan_parallel(Problem pb)
{
    const unsigned long long T = (unsigned long long)pb.grid * pb.threads;
    const int lane = threadIdx.x & 31, n = pb.n, c = pb.comps;
    const int ntop = n - 1 - pb.w, ntp = ntop > 0 ? ntop : 0;
    const unsigned long long warp = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned long long nwarps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    double xh[2 * kMaxN], xl[2 * kMaxN];  // [comps][kMaxN], per lane
    for (unsigned long long t = warp; t < T; t += nwarps) {
        if ((int)pb.tmax[t] < pb.thr_bin) continue;  // warp-uniform
        unsigned long long u0, u1;
        balanced_range(pb.units, T, t, &u0, &u1);
        unsigned long long a, b;
        balanced_range(u1 - u0, 32, lane, &a, &b);
        a += u0;
        b += u0;
        if (a >= b) continue;
        const unsigned long long g0 = gray_of(a);
        for (int part = 0; part < c; ++part) {
            const double* mt = pb.mt + (size_t)part * ntp * n;
            for (int r = 0; r < n; ++r) {
                dd x = {pb.x0_hi[part * n + r], pb.x0_lo[part * n + r]};
                for (int j = 0; j < ntop; ++j)
                    if ((g0 >> j) & 1ull) x = dd_add_d(x, mt[j * n + r]);
                xh[part * kMaxN + r] = x.hi;
                xl[part * kMaxN + r] = x.lo;
            }
        }
        for (unsigned long long u = a;;) {
            if (hist_bin(unit_bound_rt(pb, xh)) >= pb.thr_bin) {
                const unsigned long long i = atomicAdd(pb.list_n, 1ull);
                if (i < pb.list_cap) pb.list_u[i] = u;
            }
            if (++u >= b) break;
            const int j = __ffsll((long long)u) - 1;
            const bool add = (gray_of(u) >> j) & 1ull;
            for (int part = 0; part < c; ++part) {
                const double* col = pb.mt + ((size_t)part * ntp + j) * n;
                for (int r = 0; r < n; ++r) {
                    const double m = add ? col[r] : -col[r];
                    dd s = two_sum(xh[part * kMaxN + r], m);
                    dd z = fast_two_sum(s.hi, add_rn(s.lo, xl[part * kMaxN + r]));
                    xh[part * kMaxN + r] = z.hi;
                    xl[part * kMaxN + r] = z.lo;
                }
            }
        }
    }
}

// *list_bin = the lowest bin whose tail (units at or above it) holds
// at most raw_cap/2 units by bound_walk's count.
__global__ void pick_list_bin(Problem pb)
{
    __shared__ unsigned s_c[kHistBins];
    for (int i = threadIdx.x; i < kHistBins; i += blockDim.x) s_c[i] = pb.pre_cnt[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long tail = 0;
        int b = kHistBins;
        while (b > 0 && tail + s_c[b - 1] <= pb.raw_cap / 2) tail += s_c[--b];
        *pb.list_bin = b;
    }
}

// Keeps the mode-1 listed units whose bin >= thr_bin.
__global__ void collect_listed(Problem pb)
{
    const unsigned long long m = *pb.raw_n < pb.raw_cap ? *pb.raw_n : pb.raw_cap;
    for (unsigned long long e = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; e < m;
         e += (unsigned long long)gridDim.x * blockDim.x)
        if ((int)pb.raw_b[e] >= pb.thr_bin) {
            const unsigned long long i = atomicAdd(pb.list_n, 1ull);
            if (i < pb.list_cap) pb.list_u[i] = pb.raw_u[e];
        }
}

__global__ void __launch_bounds__(256) refine_real(Problem pb, unsigned long long count)
{
    extern __shared__ __align__(16) double sm[];
    const int n = pb.n, G = pb.g, terms = 1 << pb.w, nq = terms / G;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double* s_dh = sm;
    double* s_dl = s_dh + terms * n;
    double* s_x = s_dl + terms * n;      // [nwarps][2n]
    double* s_g = s_x + nwarps * 2 * n;  // [nwarps][nq]
    for (int i = threadIdx.x; i < terms * n; i += blockDim.x) {
        s_dh[i] = pb.de_hi[i];
        s_dl[i] = pb.de_lo[i];
    }
    __syncthreads();
    double* xw = s_x + wid * 2 * n;
    double* gw = s_g + wid * nq;
    dd corr = {0.0, 0.0};
    for (unsigned long long e = (unsigned long long)blockIdx.x * nwarps + wid; e < count;
         e += (unsigned long long)gridDim.x * nwarps) {
        if (pb.list_x) {
            const double* src = pb.list_x + e * (2 * n);
            for (int i = lane; i < 2 * n; i += 32) xw[i] = src[i];
        } else {
            unit_base(pb, pb.list_u[e], 0, lane, xw, xw + n);
        }
        __syncwarp();
        for (int q = lane; q < nq; q += 32) gw[q] = group_sum_real_rt(xw, s_dh + q * n * G, n, pb.na, G);
        dd acc = {0.0, 0.0};
        for (int d = lane; d < terms; d += 32) {
            const int q = d / G, i = d % G;
            int k = (q * n) * G + i;
            dd p = dd_add(dd{xw[0], xw[n]}, dd{s_dh[k], s_dl[k]});
            for (int r = 1; r < n; ++r) {
                k = (q * n + r) * G + i;
                p = dd_mul(p, dd_add(dd{xw[r], xw[n + r]}, dd{s_dh[k], s_dl[k]}));
            }
            acc = (__popc(d) & 1) ? dd_add(acc, dd_neg(p)) : dd_add(acc, p);
        }
        acc = warp_sum_dd(acc);
        __syncwarp();
        if (lane == 0) {
            double f = 0.0;
            for (int q = 0; q < nq; ++q) f = (__popc(q) & 1) ? sub_rn(f, gw[q]) : add_rn(f, gw[q]);
            dd c = dd_add_d(acc, -f);
            if (pb.list_u[e] & 1ull) c = dd_neg(c);
            corr = dd_add(corr, c);
        }
        __syncwarp();
    }
    dd tot[1] = {corr};
    grid_reduce<1>(tot, pb);
}

__global__ void __launch_bounds__(256) refine_complex(Problem pb, unsigned long long count)
{
    extern __shared__ __align__(16) double sm[];
    const int n = pb.n, G = pb.g, terms = 1 << pb.w, nq = terms / G;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double* s_dh = sm;                    // [2][terms*n]
    double* s_dl = s_dh + 2 * terms * n;  // [2][terms*n]
    double* s_x = s_dl + 2 * terms * n;   // [nwarps][4n]
    double* s_g = s_x + nwarps * 4 * n;   // [nwarps][2*nq]
    for (int i = threadIdx.x; i < 2 * terms * n; i += blockDim.x) {
        s_dh[i] = pb.de_hi[i];
        s_dl[i] = pb.de_lo[i];
    }
    __syncthreads();
    const double* drh = s_dh;
    const double* dih = s_dh + terms * n;
    const double* drl = s_dl;
    const double* dil = s_dl + terms * n;
    double* xw = s_x + wid * 4 * n;  // xr hi, xr lo, xi hi, xi lo
    double* gw = s_g + wid * 2 * nq;
    dd corr_r = {0.0, 0.0}, corr_i = {0.0, 0.0};
    for (unsigned long long e = (unsigned long long)blockIdx.x * nwarps + wid; e < count;
         e += (unsigned long long)gridDim.x * nwarps) {
        if (pb.list_x) {
            const double* src = pb.list_x + e * (4 * n);
            for (int i = lane; i < 4 * n; i += 32) xw[i] = src[i];
        } else {
            unit_base(pb, pb.list_u[e], 0, lane, xw, xw + n);
            unit_base(pb, pb.list_u[e], 1, lane, xw + 2 * n, xw + 3 * n);
        }
        __syncwarp();
        for (int q = lane; q < nq; q += 32)
            group_sum_complex_rt(xw, xw + 2 * n, drh + q * n * G, dih + q * n * G, n, G, gw[2 * q],
                                 gw[2 * q + 1]);
        dd ar = {0.0, 0.0}, ai = {0.0, 0.0};
        for (int d = lane; d < terms; d += 32) {
            const int q = d / G, i = d % G;
            int k = (q * n) * G + i;
            dd pr = dd_add(dd{xw[0], xw[n]}, dd{drh[k], drl[k]});
            dd pi = dd_add(dd{xw[2 * n], xw[3 * n]}, dd{dih[k], dil[k]});
            for (int r = 1; r < n; ++r) {
                k = (q * n + r) * G + i;
                dd yr = dd_add(dd{xw[r], xw[n + r]}, dd{drh[k], drl[k]});
                dd yi = dd_add(dd{xw[2 * n + r], xw[3 * n + r]}, dd{dih[k], dil[k]});
                dd nr = dd_add(dd_mul(pr, yr), dd_neg(dd_mul(pi, yi)));
                dd ni = dd_add(dd_mul(pr, yi), dd_mul(pi, yr));
                pr = nr;
                pi = ni;
            }
            if (__popc(d) & 1) {
                ar = dd_add(ar, dd_neg(pr));
                ai = dd_add(ai, dd_neg(pi));
            } else {
                ar = dd_add(ar, pr);
                ai = dd_add(ai, pi);
            }
        }
        ar = warp_sum_dd(ar);
        ai = warp_sum_dd(ai);
        __syncwarp();
        if (lane == 0) {
            double fr = 0.0, fi = 0.0;
            for (int q = 0; q < nq; ++q) {
                if (__popc(q) & 1) {
                    fr = sub_rn(fr, gw[2 * q]);
                    fi = sub_rn(fi, gw[2 * q + 1]);
                } else {
                    fr = add_rn(fr, gw[2 * q]);
                    fi = add_rn(fi, gw[2 * q + 1]);
                }
            }
            dd cr = dd_add_d(ar, -fr), ci = dd_add_d(ai, -fi);
            if (pb.list_u[e] & 1ull) {
                cr = dd_neg(cr);
                ci = dd_neg(ci);
            }
            corr_r = dd_add(corr_r, cr);
            corr_i = dd_add(corr_i, ci);
        }
        __syncwarp();
    }
    dd tot[2] = {corr_r, corr_i};
    grid_reduce<2>(tot, pb);
}

}  // namespace

template <int N>
int launch_bound_n(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s);

int launch_bound_pass(const Problem& pb, int blocks, cudaStream_t s)
{
    const int threads = 256;
    const size_t smem = bound_smem_bytes_f(pb.n, pb.comps, pb.w);
    // Two CTAs per SM, but at least 8 units per thread: a thread's first
    // unit base costs n*(n-1-w) adds, so few units per thread would be
    // dominated by that start.
    blocks *= 2;
    unsigned long long max_blocks = (pb.units + 8ull * threads - 1) / (8ull * threads);
    if ((unsigned long long)blocks > max_blocks) blocks = (int)max_blocks;
    if (blocks < 1) blocks = 1;
    int st = SPB_ERR_INVALID;
    switch (pb.n) {
#define SPB_CASE(N) \
    case N: st = launch_bound_n<N>(pb, blocks, threads, smem, s); break;
        SPB_FOR_EACH_N(SPB_CASE)
#undef SPB_CASE
    default:
        spb_set_error("bound pass: n=%d outside 1..%d", pb.n, kMaxN);
        return SPB_ERR_INVALID;
    }
    if (st != SPB_OK) return st;
    pick_list_bin<<<1, 128, 0, s>>>(pb);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

int launch_scan_parallel(const Problem& pb, cudaStream_t s)
{
    scan_parallel<<<pb.grid * 4, 128, 0, s>>>(pb);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

int launch_collect(const Problem& pb, cudaStream_t s)
{
    collect_listed<<<(unsigned)((pb.raw_cap + 255) / 256), 256, 0, s>>>(pb);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

size_t refine_smem_bytes(const Problem& pb, int threads)
{
    const size_t terms = (size_t)1 << pb.w, n = pb.n, c = pb.comps, nq = terms / pb.g;
    const size_t nwarps = threads / 32;
    return sizeof(double) * (2 * c * terms * n + nwarps * (2 * c * n + c * nq));
}

int launch_refine(const Problem& pb, unsigned long long count, int blocks, cudaStream_t s)
{
    const int threads = 256;
    const size_t smem = refine_smem_bytes(pb, threads);
    auto kern = pb.comps == 1 ? refine_real : refine_complex;
    int dev = 0, optin = 0;
    SPB_CUDA_TRY(cudaGetDevice(&dev));
    SPB_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    SPB_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    if (smem + fa.sharedSizeBytes > (size_t)optin) {
        spb_set_error("refine: n=%d needs %zu B shared memory", pb.n, smem);
        return SPB_ERR_INVALID;
    }
    SPB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      optin - (int)fa.sharedSizeBytes));
    kern<<<blocks, threads, smem, s>>>(pb, count);
    SPB_CUDA_TRY(cudaGetLastError());
    return SPB_OK;
}

}  // namespace dense
}  // namespace spb
