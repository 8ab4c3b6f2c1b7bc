/*
 * TEST INFRASTRUCTURE ONLY — the checker, never the product.
 *
 * CPU restatement of the reference's NW-Ryser permanent, plus exact oracles:
 *   orc_dense_nw     Algorithms/CPU/Dense/dpNaivePerman.h:46-142
 *   orc_sparse_nw    Algorithms/CPU/Sparse/spNaivePerman.h:46-172
 *                    (CSC/CSR as built by Structures/SparseMatrix.h:61-101)
 *   orc_complex_nw   Algorithms/Complex/cpuComputeComplex.h:34-142
 *   orc_binary_ryser_u128      exact plain Ryser mod 2^128 for 0/1 matrices
 *   orc_perm_mod_primes[_gauss] NW-Ryser mod p (Montgomery), for CRT
 *
 * Each NW routine follows the reference's algorithm: x_i = a_{i,n-1} -
 * rowsum_i/2, Gray-code walk over k in [1, 2^(n-1)), column ctz(k) added or
 * removed, signed product accumulated, result (4(n%2)-2)*(prod(x0)+sum).  The
 * thread split is the reference's static ceil split; partial sums are merged
 * in thread order so the oracle is deterministic (the reference uses
 * `omp atomic`, dpNaivePerman.h:135-136).
 */
#include "oracle.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

static int clamp_threads(int threads)
{
    if (threads < 1) threads = 1;
    return threads;
}

/* ---------------------------------------------------------------- dense -- */

double orc_dense_nw(const double* a, int n, int threads)
{
    threads = clamp_threads(threads);
    if (n <= 0) return 1.0;

    double* x = (double*)malloc(sizeof(double) * n);
    double* mt = (double*)malloc(sizeof(double) * n * n);
    double product = 1.0;
    /* dpNaivePerman.h:53-65 */
    for (int i = 0; i < n; ++i) {
        double rowSum = 0.0;
        for (int j = 0; j < n; ++j) rowSum += a[i * n + j];
        x[i] = a[i * n + (n - 1)] - rowSum / 2;
        product *= x[i];
    }
    double productSum = product;
    /* dpNaivePerman.h:67-74: column-major copy */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) mt[j * n + i] = a[i * n + j];

    long long start = 1, end = 1LL << (n - 1);
    double* partial = (double*)calloc((size_t)threads, sizeof(double));

#pragma omp parallel num_threads(threads)
    {
        int tid = omp_get_thread_num();
        int nth = omp_get_num_threads();
        double* myX = (double*)malloc(sizeof(double) * n);
        memcpy(myX, x, sizeof(double) * n);
        double myResult = 0.0;
        long long chunk = (end - start + nth - 1) / nth;
        long long myStart = start + tid * chunk;
        long long myEnd = myStart + chunk < end ? myStart + chunk : end;
        if (myStart < myEnd) {
            long long gray = (myStart - 1) ^ ((myStart - 1) >> 1);
            for (int j = 0; j < n - 1; ++j)
                if ((gray >> j) & 1LL)
                    for (int i = 0; i < n; ++i) myX[i] += mt[j * n + i];
            int sign = (myStart & 1LL) ? -1 : 1;
            /* dpNaivePerman.h:116-133 */
            for (long long k = myStart; k < myEnd; ++k) {
                int col = __builtin_ctzll((unsigned long long)k);
                gray ^= 1LL << col;
                double added = ((1LL << col) & gray) ? 1.0 : -1.0;
                double prod = 1.0;
                const double* c = mt + col * n;
                for (int r = 0; r < n; ++r) {
                    myX[r] += added * c[r];
                    prod *= myX[r];
                }
                myResult += sign * prod;
                sign = -sign;
            }
        }
        partial[tid] = myResult;
        free(myX);
    }
    for (int t = 0; t < threads; ++t) productSum += partial[t];
    free(partial);
    free(x);
    free(mt);
    return (4 * (n % 2) - 2) * productSum;
}

/* --------------------------------------------------------------- sparse -- */

double orc_sparse_nw(const double* a, int n, int threads)
{
    threads = clamp_threads(threads);
    if (n <= 0) return 1.0;
    int nnz = 0;
    for (int i = 0; i < n * n; ++i) nnz += a[i] != 0.0;
    /* SparseMatrix.h:61-101: CSR and CSC in ascending index order */
    int* rptrs = (int*)malloc(sizeof(int) * (n + 1));
    int* cptrs = (int*)malloc(sizeof(int) * (n + 1));
    int* rows = (int*)malloc(sizeof(int) * (nnz ? nnz : 1));
    double* rvals = (double*)malloc(sizeof(double) * (nnz ? nnz : 1));
    double* cvals = (double*)malloc(sizeof(double) * (nnz ? nnz : 1));
    int rn = 0, cn = 0;
    for (int i = 0; i < n; ++i) {
        rptrs[i] = rn;
        cptrs[i] = cn;
        for (int j = 0; j < n; ++j) {
            if (a[i * n + j] != 0.0) rvals[rn++] = a[i * n + j];
            if (a[j * n + i] != 0.0) { rows[cn] = j; cvals[cn] = a[j * n + i]; ++cn; }
        }
    }
    rptrs[n] = rn;
    cptrs[n] = cn;

    double* x = (double*)malloc(sizeof(double) * n);
    double product = 1.0;
    /* spNaivePerman.h:59-70 */
    for (int i = 0; i < n; ++i) {
        double rowSum = 0.0;
        for (int p = rptrs[i]; p < rptrs[i + 1]; ++p) rowSum += rvals[p];
        x[i] = a[i * n + (n - 1)] - rowSum / 2;
        product *= x[i];
    }
    double productSum = product;
    long long start = 1, end = 1LL << (n - 1);
    double* partial = (double*)calloc((size_t)threads, sizeof(double));

#pragma omp parallel num_threads(threads)
    {
        int tid = omp_get_thread_num();
        int nth = omp_get_num_threads();
        double* myX = (double*)malloc(sizeof(double) * n);
        memcpy(myX, x, sizeof(double) * n);
        double myResult = 0.0;
        long long chunk = (end - start + nth - 1) / nth;
        long long myStart = start + tid * chunk;
        long long myEnd = myStart + chunk < end ? myStart + chunk : end;
        if (myStart < myEnd) {
            long long gray = (myStart - 1) ^ ((myStart - 1) >> 1);
            for (int j = 0; j < n - 1; ++j)
                if ((gray >> j) & 1LL)
                    for (int p = cptrs[j]; p < cptrs[j + 1]; ++p) myX[rows[p]] += cvals[p];
            int zeros = 0;
            for (int i = 0; i < n; ++i) zeros += myX[i] == 0.0;
            int sign = (myStart & 1LL) ? -1 : 1;
            /* spNaivePerman.h:124-165 */
            for (long long k = myStart; k < myEnd; ++k) {
                int col = __builtin_ctzll((unsigned long long)k);
                gray ^= 1LL << col;
                double added = ((1LL << col) & gray) ? 1.0 : -1.0;
                for (int p = cptrs[col]; p < cptrs[col + 1]; ++p) {
                    int r = rows[p];
                    double v = myX[r];
                    if (v == 0.0) --zeros;
                    v += added * cvals[p];
                    if (v == 0.0) ++zeros;
                    myX[r] = v;
                }
                if (zeros == 0) {
                    double prod = 1.0;
                    for (int r = 0; r < n; ++r) prod *= myX[r];
                    myResult += sign * prod;
                }
                sign = -sign;
            }
        }
        partial[tid] = myResult;
        free(myX);
    }
    for (int t = 0; t < threads; ++t) productSum += partial[t];
    free(partial);
    free(x);
    free(rptrs);
    free(cptrs);
    free(rows);
    free(rvals);
    free(cvals);
    return (4 * (n % 2) - 2) * productSum;
}

/* -------------------------------------------------------------- complex -- */

void orc_complex_nw(const double* a, int n, int threads, double* out_re, double* out_im)
{
    threads = clamp_threads(threads);
    if (n <= 0) { *out_re = 1.0; *out_im = 0.0; return; }
    double* xr = (double*)malloc(sizeof(double) * n);
    double* xi = (double*)malloc(sizeof(double) * n);
    double* mr = (double*)malloc(sizeof(double) * n * n);
    double* mi = (double*)malloc(sizeof(double) * n * n);
    double pr = 1.0, pi = 0.0;
    /* cpuComputeComplex.h:40-51 */
    for (int i = 0; i < n; ++i) {
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < n; ++j) { sr += a[2 * (i * n + j)]; si += a[2 * (i * n + j) + 1]; }
        xr[i] = a[2 * (i * n + n - 1)] - sr / 2;
        xi[i] = a[2 * (i * n + n - 1) + 1] - si / 2;
        double tr = pr * xr[i] - pi * xi[i];
        double ti = pr * xi[i] + pi * xr[i];
        pr = tr;
        pi = ti;
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            mr[j * n + i] = a[2 * (i * n + j)];
            mi[j * n + i] = a[2 * (i * n + j) + 1];
        }
    double sumr = pr, sumi = pi;
    long long start = 1, end = 1LL << (n - 1);
    double* part = (double*)calloc((size_t)threads * 2, sizeof(double));

#pragma omp parallel num_threads(threads)
    {
        int tid = omp_get_thread_num();
        int nth = omp_get_num_threads();
        double* yr = (double*)malloc(sizeof(double) * n);
        double* yi = (double*)malloc(sizeof(double) * n);
        memcpy(yr, xr, sizeof(double) * n);
        memcpy(yi, xi, sizeof(double) * n);
        double accr = 0.0, acci = 0.0;
        long long chunk = (end - start + nth - 1) / nth;
        long long myStart = start + tid * chunk;
        long long myEnd = myStart + chunk < end ? myStart + chunk : end;
        if (myStart < myEnd) {
            long long gray = (myStart - 1) ^ ((myStart - 1) >> 1);
            for (int j = 0; j < n - 1; ++j)
                if ((gray >> j) & 1LL)
                    for (int i = 0; i < n; ++i) { yr[i] += mr[j * n + i]; yi[i] += mi[j * n + i]; }
            double sign = (myStart & 1LL) ? -1.0 : 1.0;
            /* cpuComputeComplex.h:98-115 */
            for (long long k = myStart; k < myEnd; ++k) {
                int col = __builtin_ctzll((unsigned long long)k);
                gray ^= 1LL << col;
                double added = ((1LL << col) & gray) ? 1.0 : -1.0;
                double qr = 1.0, qi = 0.0;
                for (int r = 0; r < n; ++r) {
                    yr[r] += added * mr[col * n + r];
                    yi[r] += added * mi[col * n + r];
                    double tr = qr * yr[r] - qi * yi[r];
                    double ti = qr * yi[r] + qi * yr[r];
                    qr = tr;
                    qi = ti;
                }
                accr += sign * qr;
                acci += sign * qi;
                sign = -sign;
            }
        }
        part[2 * tid] = accr;
        part[2 * tid + 1] = acci;
        free(yr);
        free(yi);
    }
    for (int t = 0; t < threads; ++t) { sumr += part[2 * t]; sumi += part[2 * t + 1]; }
    free(part);
    double f = (double)(4 * (n % 2) - 2);
    *out_re = f * sumr;
    *out_im = f * sumi;
    free(xr);
    free(xi);
    free(mr);
    free(mi);
}

/* ------------------------------------------------------- binary (exact) -- */

void orc_binary_ryser_u128(const uint8_t* a, int n, int threads, uint64_t out[2])
{
    threads = clamp_threads(threads);
    if (n <= 0) { out[0] = 1; out[1] = 0; return; }
    long long end = 1LL << n; /* all 2^n subsets; subset 0 contributes 0 */
    u128* part = (u128*)calloc((size_t)threads, sizeof(u128));
    uint8_t* mt = (uint8_t*)malloc((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) mt[j * n + i] = a[i * n + j] ? 1 : 0;

#pragma omp parallel num_threads(threads)
    {
        int tid = omp_get_thread_num();
        int nth = omp_get_num_threads();
        int x[64];
        memset(x, 0, sizeof(x));
        u128 acc = 0;
        long long chunk = (end - 1 + nth - 1) / nth;
        long long myStart = 1 + tid * chunk;
        long long myEnd = myStart + chunk < end ? myStart + chunk : end;
        if (myStart < myEnd) {
            long long gray = (myStart - 1) ^ ((myStart - 1) >> 1);
            for (int j = 0; j < n; ++j)
                if ((gray >> j) & 1LL)
                    for (int i = 0; i < n; ++i) x[i] += mt[j * n + i];
            for (long long k = myStart; k < myEnd; ++k) {
                int col = __builtin_ctzll((unsigned long long)k);
                gray ^= 1LL << col;
                int d = ((gray >> col) & 1LL) ? 1 : -1;
                const uint8_t* c = mt + col * n;
                u128 prod = 1;
                for (int r = 0; r < n; ++r) {
                    x[r] += d * c[r];
                    prod *= (u128)(uint64_t)x[r];
                }
                /* |S| parity of gray(k) equals k & 1 */
                if (k & 1LL) acc -= prod; else acc += prod;
            }
        }
        part[tid] = acc;
    }
    u128 total = 0;
    for (int t = 0; t < threads; ++t) total += part[t];
    if (n & 1) total = (u128)0 - total;
    out[0] = (uint64_t)total;
    out[1] = (uint64_t)(total >> 64);
    free(part);
    free(mt);
}

/* ------------------------------------------------------ modular (exact) -- */

typedef struct {
    uint64_t p, pinv, r2; /* pinv = -p^{-1} mod 2^64, r2 = 2^128 mod p */
} mont_t;

static mont_t mont_init(uint64_t p)
{
    mont_t m;
    m.p = p;
    uint64_t inv = 1; /* Newton iteration for p^{-1} mod 2^64 */
    for (int i = 0; i < 7; ++i) inv *= 2 - p * inv;
    m.pinv = (uint64_t)0 - inv;
    u128 r = ((u128)1 << 64) % p;
    m.r2 = (uint64_t)((r * r) % p);
    return m;
}

static inline uint64_t mont_mul(const mont_t* m, uint64_t a, uint64_t b)
{
    u128 t = (u128)a * b;
    uint64_t k = (uint64_t)t * m->pinv;
    u128 u = (t + (u128)k * m->p) >> 64;
    uint64_t r = (uint64_t)u;
    return r >= m->p ? r - m->p : r;
}

static inline uint64_t addm(uint64_t a, uint64_t b, uint64_t p)
{
    uint64_t s = a + b;
    return s >= p ? s - p : s;
}

static inline uint64_t subm(uint64_t a, uint64_t b, uint64_t p)
{
    return a >= b ? a - b : a + p - b;
}

static inline uint64_t to_mont(const mont_t* m, uint64_t a) { return mont_mul(m, a % m->p, m->r2); }
static inline uint64_t from_mont(const mont_t* m, uint64_t a) { return mont_mul(m, a, 1); }

#define CHUNKS_PER_PRIME 64

/* One Gray range [ks, ke) of the NW sum mod p: returns the signed partial sum
 * in Montgomery form.  kt is the transposed Montgomery-form matrix, x0 the
 * Montgomery-form NW start vector. */
static uint64_t mod_range(const mont_t* m, const uint64_t* kt, const uint64_t* x0, int n,
                          long long ks, long long ke)
{
    uint64_t p = m->p;
    uint64_t x[64];
    memcpy(x, x0, sizeof(uint64_t) * n);
    long long gray = (ks - 1) ^ ((ks - 1) >> 1);
    for (int j = 0; j < n - 1; ++j)
        if ((gray >> j) & 1LL)
            for (int i = 0; i < n; ++i) x[i] = addm(x[i], kt[j * n + i], p);
    uint64_t acc = 0;
    for (long long k = ks; k < ke; ++k) {
        int col = __builtin_ctzll((unsigned long long)k);
        gray ^= 1LL << col;
        const uint64_t* c = kt + col * n;
        if ((gray >> col) & 1LL)
            for (int r = 0; r < n; ++r) x[r] = addm(x[r], c[r], p);
        else
            for (int r = 0; r < n; ++r) x[r] = subm(x[r], c[r], p);
        /* two independent product chains for ILP */
        uint64_t pa = x[0], pb = n > 1 ? x[1] : to_mont(m, 1);
        int r = 2;
        for (; r + 1 < n; r += 2) {
            pa = mont_mul(m, pa, x[r]);
            pb = mont_mul(m, pb, x[r + 1]);
        }
        if (r < n) pa = mont_mul(m, pa, x[r]);
        uint64_t prod = mont_mul(m, pa, pb);
        acc = (k & 1LL) ? subm(acc, prod, p) : addm(acc, prod, p);
    }
    return acc;
}

void orc_perm_mod_primes(const uint64_t* kmod, int n, const uint64_t* primes, int np,
                         int threads, uint64_t* out)
{
    threads = clamp_threads(threads);
    if (n <= 0) { for (int q = 0; q < np; ++q) out[q] = 1 % primes[q]; return; }
    long long end = 1LL << (n - 1);
    int nchunks = end >= CHUNKS_PER_PRIME ? CHUNKS_PER_PRIME : (int)end;
    uint64_t* kt = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)np * n * n);
    uint64_t* x0 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)np * n);
    uint64_t* base = (uint64_t*)malloc(sizeof(uint64_t) * np);
    uint64_t* part = (uint64_t*)calloc((size_t)np * nchunks, sizeof(uint64_t));
    for (int q = 0; q < np; ++q) {
        mont_t m = mont_init(primes[q]);
        uint64_t p = m.p, inv2m = to_mont(&m, (p + 1) / 2);
        const uint64_t* K = kmod + (size_t)q * n * n;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) kt[(size_t)q * n * n + j * n + i] = to_mont(&m, K[i * n + j]);
        uint64_t prod = to_mont(&m, 1);
        for (int i = 0; i < n; ++i) {
            uint64_t rs = 0;
            for (int j = 0; j < n; ++j) rs = addm(rs, kt[(size_t)q * n * n + j * n + i], p);
            uint64_t xi = subm(kt[(size_t)q * n * n + (n - 1) * n + i], mont_mul(&m, rs, inv2m), p);
            x0[(size_t)q * n + i] = xi;
            prod = mont_mul(&m, prod, xi);
        }
        base[q] = prod;
    }
    long long span = end - 1;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
    for (long long t = 0; t < (long long)np * nchunks; ++t) {
        int q = (int)(t / nchunks), c = (int)(t % nchunks);
        mont_t m = mont_init(primes[q]);
        long long ks = 1 + span * c / nchunks, ke = 1 + span * (c + 1) / nchunks;
        part[t] = ks < ke ? mod_range(&m, kt + (size_t)q * n * n, x0 + (size_t)q * n, n, ks, ke) : 0;
    }
    for (int q = 0; q < np; ++q) {
        mont_t m = mont_init(primes[q]);
        uint64_t s = base[q];
        for (int c = 0; c < nchunks; ++c) s = addm(s, part[(size_t)q * nchunks + c], m.p);
        uint64_t two = to_mont(&m, 2);
        s = mont_mul(&m, s, two);
        if (n % 2 == 0) s = subm(0, s, m.p); /* factor 4(n%2)-2 = +2 (odd n) or -2 (even n) */
        out[q] = from_mont(&m, s);
    }
    free(kt);
    free(x0);
    free(base);
    free(part);
}

static uint64_t gauss_range(const mont_t* m, const uint64_t* ktr, const uint64_t* kti,
                            const uint64_t* x0r, const uint64_t* x0i, int n, long long ks,
                            long long ke, uint64_t* acc_im)
{
    uint64_t p = m->p;
    uint64_t xr[64], xi[64];
    memcpy(xr, x0r, sizeof(uint64_t) * n);
    memcpy(xi, x0i, sizeof(uint64_t) * n);
    long long gray = (ks - 1) ^ ((ks - 1) >> 1);
    for (int j = 0; j < n - 1; ++j)
        if ((gray >> j) & 1LL)
            for (int i = 0; i < n; ++i) {
                xr[i] = addm(xr[i], ktr[j * n + i], p);
                xi[i] = addm(xi[i], kti[j * n + i], p);
            }
    uint64_t one = to_mont(m, 1);
    uint64_t ar = 0, ai = 0;
    for (long long k = ks; k < ke; ++k) {
        int col = __builtin_ctzll((unsigned long long)k);
        gray ^= 1LL << col;
        const uint64_t* cr = ktr + col * n;
        const uint64_t* ci = kti + col * n;
        if ((gray >> col) & 1LL)
            for (int r = 0; r < n; ++r) { xr[r] = addm(xr[r], cr[r], p); xi[r] = addm(xi[r], ci[r], p); }
        else
            for (int r = 0; r < n; ++r) { xr[r] = subm(xr[r], cr[r], p); xi[r] = subm(xi[r], ci[r], p); }
        uint64_t qr = one, qi = 0;
        for (int r = 0; r < n; ++r) {
            uint64_t tr = subm(mont_mul(m, qr, xr[r]), mont_mul(m, qi, xi[r]), p);
            uint64_t ti = addm(mont_mul(m, qr, xi[r]), mont_mul(m, qi, xr[r]), p);
            qr = tr;
            qi = ti;
        }
        if (k & 1LL) { ar = subm(ar, qr, p); ai = subm(ai, qi, p); }
        else { ar = addm(ar, qr, p); ai = addm(ai, qi, p); }
    }
    *acc_im = ai;
    return ar;
}

void orc_perm_mod_primes_gauss(const uint64_t* kre, const uint64_t* kim, int n,
                               const uint64_t* primes, int np, int threads,
                               uint64_t* out_re, uint64_t* out_im)
{
    threads = clamp_threads(threads);
    if (n <= 0) {
        for (int q = 0; q < np; ++q) { out_re[q] = 1 % primes[q]; out_im[q] = 0; }
        return;
    }
    long long end = 1LL << (n - 1);
    int nchunks = end >= CHUNKS_PER_PRIME ? CHUNKS_PER_PRIME : (int)end;
    size_t nn = (size_t)n * n;
    uint64_t* ktr = (uint64_t*)malloc(sizeof(uint64_t) * np * nn);
    uint64_t* kti = (uint64_t*)malloc(sizeof(uint64_t) * np * nn);
    uint64_t* x0r = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)np * n);
    uint64_t* x0i = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)np * n);
    uint64_t* br = (uint64_t*)malloc(sizeof(uint64_t) * np);
    uint64_t* bi = (uint64_t*)malloc(sizeof(uint64_t) * np);
    uint64_t* pr_ = (uint64_t*)calloc((size_t)np * nchunks, sizeof(uint64_t));
    uint64_t* pi_ = (uint64_t*)calloc((size_t)np * nchunks, sizeof(uint64_t));
    for (int q = 0; q < np; ++q) {
        mont_t m = mont_init(primes[q]);
        uint64_t p = m.p, inv2m = to_mont(&m, (p + 1) / 2);
        const uint64_t* Kr = kre + q * nn;
        const uint64_t* Ki = kim + q * nn;
        uint64_t* tr = ktr + q * nn;
        uint64_t* ti = kti + q * nn;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                tr[j * n + i] = to_mont(&m, Kr[i * n + j]);
                ti[j * n + i] = to_mont(&m, Ki[i * n + j]);
            }
        uint64_t qr = to_mont(&m, 1), qi = 0;
        for (int i = 0; i < n; ++i) {
            uint64_t sr = 0, si = 0;
            for (int j = 0; j < n; ++j) { sr = addm(sr, tr[j * n + i], p); si = addm(si, ti[j * n + i], p); }
            uint64_t vr = subm(tr[(n - 1) * n + i], mont_mul(&m, sr, inv2m), p);
            uint64_t vi = subm(ti[(n - 1) * n + i], mont_mul(&m, si, inv2m), p);
            x0r[(size_t)q * n + i] = vr;
            x0i[(size_t)q * n + i] = vi;
            uint64_t nr = subm(mont_mul(&m, qr, vr), mont_mul(&m, qi, vi), p);
            uint64_t ni = addm(mont_mul(&m, qr, vi), mont_mul(&m, qi, vr), p);
            qr = nr;
            qi = ni;
        }
        br[q] = qr;
        bi[q] = qi;
    }
    long long span = end - 1;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
    for (long long t = 0; t < (long long)np * nchunks; ++t) {
        int q = (int)(t / nchunks), c = (int)(t % nchunks);
        mont_t m = mont_init(primes[q]);
        long long ks = 1 + span * c / nchunks, ke = 1 + span * (c + 1) / nchunks;
        uint64_t im = 0;
        pr_[t] = ks < ke ? gauss_range(&m, ktr + q * nn, kti + q * nn, x0r + (size_t)q * n,
                                       x0i + (size_t)q * n, n, ks, ke, &im)
                         : 0;
        pi_[t] = im;
    }
    for (int q = 0; q < np; ++q) {
        mont_t m = mont_init(primes[q]);
        uint64_t sr = br[q], si = bi[q];
        for (int c = 0; c < nchunks; ++c) {
            sr = addm(sr, pr_[(size_t)q * nchunks + c], m.p);
            si = addm(si, pi_[(size_t)q * nchunks + c], m.p);
        }
        uint64_t two = to_mont(&m, 2);
        sr = mont_mul(&m, sr, two);
        si = mont_mul(&m, si, two);
        if (n % 2 == 0) { sr = subm(0, sr, m.p); si = subm(0, si, m.p); }
        out_re[q] = from_mont(&m, sr);
        out_im[q] = from_mont(&m, si);
    }
    free(ktr); free(kti); free(x0r); free(x0i); free(br); free(bi); free(pr_); free(pi_);
}

/* ------------------------------------------------------------------------
 * Sequential importance sampling (aspSingleGPU / rasmussenScaleAB,
 * Algorithms/GPU/Sparse/ApproximateSparseKernelDefinitions.cuh:32-290).
 * ---------------------------------------------------------------------- */
void orc_rasmussen_init(int n, const int* rptr, const int* col, const int* cptr, const int* row,
                        float* rv, float* cv)
{
    for (int i = 0; i < n; ++i) rv[i] = cv[i] = 1.0f;
    for (int it = 0; it < 50; ++it) {  /* ApproximateSparseKernelDefinitions.cuh:32-61 */
        for (int j = 0; j < n; ++j) {
            float s = 0.0f;
            for (int q = cptr[j]; q < cptr[j + 1]; ++q) s = s + rv[row[q]];
            cv[j] = 1.0f / s;
        }
        for (int i = 0; i < n; ++i) {
            float s = 0.0f;
            for (int p = rptr[i]; p < rptr[i + 1]; ++p) s = s + cv[col[p]];
            rv[i] = 1.0f / s;
        }
    }
}

static uint64_t orc_splitmix(uint64_t* s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* :124-172: removal of line `start` (a column when by_col) lowers the entry
 * counts of the crossing lines still present; a crossing line left with one
 * entry is matched to it; none left: no perfect matching (returns 1). */
static int orc_propagate(const int* optr, const int* oidx, const int* sptr, const int* sidx,
                         float* so, float* ss, int* cnt, int* stk, int start)
{
    int sp = 1;
    stk[0] = start;
    for (int ii = 0; ii < sp; ++ii) {
        const int j = stk[ii];
        for (int q = optr[j]; q < optr[j + 1]; ++q) {
            const int i = oidx[q];
            if (so[i] == 0.0f) continue;
            const int k = --cnt[i];
            if (k == 0) return 1;
            if (k != 1) continue;
            for (int p = sptr[i]; p < sptr[i + 1]; ++p) {
                const int j2 = sidx[p];
                if (ss[j2] == 0.0f) continue;
                so[i] = 0.0f;
                ss[j2] = 0.0f;
                stk[sp++] = j2;
                break;
            }
        }
    }
    return 0;
}

static double orc_rasmussen_one(int n, const int* rptr, const int* col, const int* cptr, const int* row,
                                const float* rv0, const float* cv0, uint64_t seed, uint64_t k,
                                float* rv, float* cv, int* re, int* ce, int* stk)
{
    for (int i = 0; i < n; ++i) {
        re[i] = rptr[i + 1] - rptr[i];
        ce[i] = cptr[i + 1] - cptr[i];
        rv[i] = rv0[i];
        cv[i] = cv0[i];
    }
    uint64_t rng = seed ^ (k * 0xD1B54A32D192ED03ull);
    double est = 1.0;
    for (int i = 0; i < n; ++i) {
        for (int it = 0; it < 10; ++it) {  /* scaleAB, :63-122 */
            for (int p = rptr[i]; p < rptr[i + 1]; ++p) {
                const int j = col[p];
                if (cv[j] == 0.0f) continue;
                float s = 0.0f;
                for (int q = cptr[j]; q < cptr[j + 1]; ++q) s = s + rv[row[q]];
                if (s == 0.0f) return 0.0;
                cv[j] = 1.0f / s;
            }
            if (rv[i] != 0.0f) {
                float s = 0.0f;
                for (int p = rptr[i]; p < rptr[i + 1]; ++p) s = s + cv[col[p]];
                if (s == 0.0f) return 0.0;
                rv[i] = 1.0f / s;
            }
        }
        const float ri = rv[i];
        if (ri == 0.0f) continue;
        const float u = (float)((orc_splitmix(&rng) >> 40) + 1ull) * 0x1p-24f;
        float run = 0.0f, prob = 0.0f;
        int chosen = -1;
        for (int p = rptr[i]; p < rptr[i + 1]; ++p) {  /* :246-259 */
            const int j = col[p];
            const float cj = cv[j];
            if (cj == 0.0f) continue;
            prob = ri * cj;
            run = run + prob;
            chosen = j;
            if (run > u) break;
        }
        if (chosen < 0) return 0.0;
        est = est * (1.0 / (double)prob);
        rv[i] = 0.0f;
        cv[chosen] = 0.0f;
        if (orc_propagate(cptr, row, rptr, col, rv, cv, re, stk, chosen) ||
            orc_propagate(rptr, col, cptr, row, cv, rv, ce, stk, i))
            return 0.0;
    }
    return est;
}

void orc_rasmussen_samples(int n, const int* rptr, const int* col, const int* cptr, const int* row,
                           const float* rv0, const float* cv0, uint64_t seed, uint64_t first,
                           uint64_t count, int threads, double* out)
{
    if (threads < 1) threads = 1;
#pragma omp parallel num_threads(threads)
    {
        float* rv = (float*)malloc(sizeof(float) * (size_t)n * 2);
        int* ib = (int*)malloc(sizeof(int) * (size_t)n * 3);
#pragma omp for schedule(static)
        for (long long k = 0; k < (long long)count; ++k)
            out[k] = orc_rasmussen_one(n, rptr, col, cptr, row, rv0, cv0, seed, first + (uint64_t)k, rv, rv + n,
                                       ib, ib + n, ib + 2 * (size_t)n);
        free(rv);
        free(ib);
    }
}
