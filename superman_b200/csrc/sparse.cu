// Sparse real permanents: spb_perm_sparse_f64.
//
// Reference behaviour: spSingleGPU (Algorithms/GPU/Sparse/spSingleGPU.cuh:
// 45-234) walks the Nijenhuis–Wilf Gray code over the compressed-column form
// of the matrix (Structures/SparseMatrix.h:61-101), updating only the flipped
// column's nonzeros (Algorithms/CPU/Sparse/spNaivePerman.h:116-162); for
// large, less sparse matrices the reference instead generates a kernel
// specialised to the matrix (Algorithms/GPU/CodeGeneration/KernelGenerator.cuh:
// 114-176, with the register-area heuristic of
// UTOrderedKernelCodeGen.cuh:68-118).
//
// Here the matrix is permuted (rows and columns; the permanent is invariant)
// so that a few "low" columns touch as few rows as possible, and the
// row-compacted walk (sparse_impl.cuh) is compiled for the resulting number of
// active rows NA: each Gray term costs 2*NA FP64 operations, the rows outside
// the low columns' support enter once per unit.  A cost model picks w (the
// number of low columns) and whether the compacted walk beats the dense walk
// at all; otherwise the dense walk runs.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dense_host.h"
#include "dense_launch.cuh"
#include "sparse_impl.cuh"

namespace spb {
namespace dense {

int choose_unit_bits(int n, int comps, const spb_options* opt);

template <int NA>
int launch_sparse_na(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s);

int launch_walk_sparse(const Problem& pb, int blocks, int threads, size_t smem, cudaStream_t s)
{
    switch (pb.na) {
#define SPB_CASE(K) \
    case K: return launch_sparse_na<K>(pb, blocks, threads, smem, s);
        SPB_CASE(1) SPB_CASE(2) SPB_CASE(3) SPB_CASE(4) SPB_CASE(5) SPB_CASE(6) SPB_CASE(7) SPB_CASE(8)
        SPB_CASE(9) SPB_CASE(10) SPB_CASE(11) SPB_CASE(12) SPB_CASE(13) SPB_CASE(14) SPB_CASE(15)
        SPB_CASE(16) SPB_CASE(17) SPB_CASE(18) SPB_CASE(19) SPB_CASE(20) SPB_CASE(21) SPB_CASE(22)
        SPB_CASE(23) SPB_CASE(24) SPB_CASE(25) SPB_CASE(26) SPB_CASE(27) SPB_CASE(28) SPB_CASE(29)
        SPB_CASE(30) SPB_CASE(31) SPB_CASE(32)
#undef SPB_CASE
    default:
        spb_set_error("row-compacted walk: %d active rows outside 1..%d", pb.na, kMaxActive);
        return SPB_ERR_INVALID;
    }
}

namespace {

int popc(unsigned long long x) { return __builtin_popcountll(x); }

// Estimated FP64-pipe operations of a walk over 2^(n-1) terms in units of
// 2^w terms.  Per term: the x additions and products of the varying rows plus
// the group combine; per unit: the double-double base update of the varying
// rows, the product of the constant rows, the inactive nonzeros of the
// flipped column (expected count `flip`), and bookkeeping.  The double-double
// mode's first pass adds a squared-term accumulation per term and the unit
// bound with its histogram update per unit.
double walk_cost(int n, int w, int na, double flip, bool dd)
{
    const double units = std::ldexp(1.0, n - 1 - w), terms = std::ldexp(1.0, w);
    const double per_term = 2.0 * na + 0.75 + (dd ? 1.0 : 0.0);
    const double per_unit = 12.0 * na + 2.0 * (n - na) + 14.0 * flip + 40.0 + (dd ? 6.0 * na + 60.0 : 0.0);
    return units * (terms * per_term + per_unit);
}

struct Choice {
    int na = 0, w = 0;
    double cost = INFINITY;
    std::vector<int> rows, cols;  // new order: position -> original index
};

// Greedy choice of the low columns: for every candidate last column, add the
// column that grows the union of row supports least (ties: fewer nonzeros,
// then lower index), and price every prefix length w.  High columns are
// ordered by ascending count of nonzeros outside the union, since the Gray
// code flips high column j once every 2^(j+1) units.
void choose(const std::vector<unsigned long long>& cm, int n, int min_ntop, bool dd, Choice* best)
{
    // The low-column table obeys the dense walk's 64 KB budget (2^w n
    // doubles), so the refinement kernel can hold it, hi and lo, in shared
    // memory.
    int wmax = std::min(10, n - 1 - min_ntop);
    while (wmax > 2 && ((size_t)1 << wmax) * (size_t)n * sizeof(double) > (size_t)64 * 1024) --wmax;
    std::vector<int> high(n), key(n), start(n + 2);
    std::vector<char> used(n);
    std::vector<int> low;
    for (int last = 0; last < n; ++last) {
        std::fill(used.begin(), used.end(), 0);
        used[last] = 1;
        low.clear();
        unsigned long long U = 0;
        for (int w = 1; w <= wmax; ++w) {
            int bj = -1, bu = 1 << 30, bc = 1 << 30;
            for (int c = 0; c < n; ++c) {
                if (used[c]) continue;
                const int u = popc(U | cm[c]), cc = popc(cm[c]);
                if (u < bu || (u == bu && cc < bc)) { bu = u; bc = cc; bj = c; }
            }
            if (bj < 0) break;
            used[bj] = 1;
            low.push_back(bj);
            U |= cm[bj];
            const int na = popc(U);
            if (w < 2 || na < 1 || na >= n || na > kMaxActive) continue;
            // the unused columns by ascending count of nonzeros outside U,
            // ties by index (a stable counting sort: keys are at most n)
            std::fill(start.begin(), start.end(), 0);
            for (int c = 0; c < n; ++c)
                if (!used[c]) {
                    key[c] = popc(cm[c] & ~U);
                    ++start[key[c] + 1];
                }
            for (int k = 0; k <= n; ++k) start[k + 1] += start[k];
            const int nh = start[n + 1];
            for (int c = 0; c < n; ++c)
                if (!used[c]) high[start[key[c]]++] = c;
            double flip = 0.0;
            for (int j = 0; j < nh; ++j) flip += std::ldexp((double)key[high[j]], -j - 1);
            const double cost = walk_cost(n, w, na, flip, dd);
            if (cost < best->cost) {
                best->cost = cost;
                best->na = na;
                best->w = w;
                best->cols = low;
                best->cols.insert(best->cols.end(), high.begin(), high.begin() + nh);
                best->cols.push_back(last);
                best->rows.clear();
                for (int r = 0; r < n; ++r)
                    if ((U >> r) & 1ull) best->rows.push_back(r);
                for (int r = 0; r < n; ++r)
                    if (!((U >> r) & 1ull)) best->rows.push_back(r);
            }
        }
    }
}

// Whether the row-compacted walk runs for matrix a under sparse_walk `mode`,
// and its plan in *ch.
bool plan_compacted(const double* a, int n, int mode, const spb_options& opt, Choice* ch)
{
    const int min_n = mode == SPB_SPARSE_WALK_ALWAYS ? 4 : 20;
    if (mode == SPB_SPARSE_WALK_NEVER || n < min_n || n > kMaxN) return false;
    std::vector<unsigned long long> cm(n, 0ull);
    for (int c = 0; c < n; ++c) {
        for (int r = 0; r < n; ++r)
            if (a[(size_t)r * n + c] != 0.0) cm[c] |= 1ull << r;
        if (cm[c] == 0ull) return false;  // zero column: the dense walk returns 0
    }
    const int min_ntop = mode == SPB_SPARSE_WALK_ALWAYS ? std::min(14, n - 3) : 14;
    const bool dd = opt.precision == SPB_PREC_DD;
    choose(cm, n, min_ntop, dd, ch);
    if (ch->na <= 0) return false;
    const int wd = choose_unit_bits(n, 1, &opt);
    return mode == SPB_SPARSE_WALK_ALWAYS || ch->cost < 0.8 * walk_cost(n, wd, n, 0.0, dd);
}

}  // namespace

int run_real_host(const double* a, int n, const spb_options* opt, spb_result* out, DeviceContext* ctx)
{
    if (a && n >= 1 && n <= kMaxN && opt->sparse_walk != SPB_SPARSE_WALK_NEVER) {
        bool has_zero = false;
        for (size_t i = 0; i < (size_t)n * n && !has_zero; ++i) has_zero = a[i] == 0.0;
        Choice ch;
        if (has_zero && plan_compacted(a, n, opt->sparse_walk, *opt, &ch)) {
            std::vector<double> ap((size_t)n * n);
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) ap[(size_t)i * n + j] = a[(size_t)ch.rows[i] * n + ch.cols[j]];
            WalkPlan plan{ch.na, ch.w};
            return run(ap.data(), false, n, 1, opt, out, &plan, ctx);
        }
    }
    return run(a, false, n, 1, opt, out, nullptr, ctx);
}

}  // namespace dense
}  // namespace spb

extern "C" int spb_sparse_plan(const double* a, int n, int mode, int* na, int* w, int* row_order,
                               int* col_order)
{
    using namespace spb::dense;
    if (!a || !na || !w || n < 1 || n > kMaxN) {
        spb_set_error("spb_sparse_plan: null argument or n outside 1..%d", kMaxN);
        return SPB_ERR_INVALID;
    }
    spb_options opt;
    spb_default_options(&opt);
    Choice ch;
    if (plan_compacted(a, n, mode, opt, &ch)) {
        *na = ch.na;
        *w = ch.w;
        for (int i = 0; i < n; ++i) {
            if (row_order) row_order[i] = ch.rows[i];
            if (col_order) col_order[i] = ch.cols[i];
        }
    } else {
        *na = n;
        *w = choose_unit_bits(n, 1, &opt);
        for (int i = 0; i < n; ++i) {
            if (row_order) row_order[i] = i;
            if (col_order) col_order[i] = i;
        }
    }
    return SPB_OK;
}

extern "C" int spb_perm_sparse_f64(const int* cptrs, const int* rows, const double* cvals, int n,
                                   const spb_options* opt_in, spb_result* out)
{
    using namespace spb::dense;
    if (!out) {
        spb_set_error("null result pointer");
        return SPB_ERR_INVALID;
    }
    std::memset(out, 0, sizeof(*out));
    if (!cptrs || n < 1 || n > kMaxN) {
        spb_set_error("spb_perm_sparse_f64: needs column pointers and 1 <= n <= %d (got n=%d)", kMaxN, n);
        return out->status = SPB_ERR_INVALID;
    }
    const int nnz = cptrs[n];
    if (cptrs[0] != 0 || nnz < 0 || (nnz > 0 && (!rows || !cvals))) {
        spb_set_error("spb_perm_sparse_f64: malformed compressed-column arrays");
        return out->status = SPB_ERR_INVALID;
    }
    for (int c = 0; c < n; ++c)
        if (cptrs[c + 1] < cptrs[c]) {
            spb_set_error("spb_perm_sparse_f64: column pointers decrease at column %d", c);
            return out->status = SPB_ERR_INVALID;
        }
    std::vector<double> a((size_t)n * n, 0.0);
    for (int c = 0; c < n; ++c) {
        for (int p = cptrs[c]; p < cptrs[c + 1]; ++p) {
            if (rows[p] < 0 || rows[p] >= n) {
                spb_set_error("spb_perm_sparse_f64: row index %d out of range in column %d", rows[p], c);
                return out->status = SPB_ERR_INVALID;
            }
            a[(size_t)rows[p] * n + c] += cvals[p];
        }
    }
    spb_options opt;
    if (opt_in) opt = *opt_in; else spb_default_options(&opt);

    return run_real_host(a.data(), n, &opt, out);
}
