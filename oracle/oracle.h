/*
 * TEST INFRASTRUCTURE ONLY — the checker, never the product.
 *
 * CPU restatement of the reference's Nijenhuis–Wilf (NW) Ryser permanent
 * (dense, sparse, complex), an exact int128 plain-Ryser for 0/1 matrices and
 * a modular NW-Ryser used to build exact rational permanents by CRT.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library.  Reference file:line citations are relative to the
 * SUPerman source tree.
 */
#ifndef SUPB_ORACLE_H
#define SUPB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Algorithms/CPU/Dense/dpNaivePerman.h:46-142.  Row-major a[n*n].  The
 * reference merges thread partials with `omp atomic` (non-deterministic
 * order); this restatement merges them in thread order. */
double orc_dense_nw(const double* a, int n, int threads);

/* Algorithms/CPU/Sparse/spNaivePerman.h:46-172 over the CSC/CSR arrays that
 * Structures/SparseMatrix.h:61-101 builds from the dense row-major a[n*n]
 * (the caller applies any column ordering first). */
double orc_sparse_nw(const double* a, int n, int threads);

/* Algorithms/Complex/cpuComputeComplex.h:34-142.  a_ri is row-major
 * interleaved (re, im) pairs: 2*n*n doubles. */
void orc_complex_nw(const double* a_ri, int n, int threads, double* re, double* im);

/* Exact plain Ryser for a 0/1 matrix (a[n*n] bytes, nonzero = 1), product and
 * signed sum in wrap-around arithmetic mod 2^128.  Exact iff |perm| < 2^127.
 * out[0] = low 64 bits, out[1] = high 64 bits (two's complement). */
void orc_binary_ryser_u128(const uint8_t* a, int n, int threads, uint64_t out[2]);

/* perm(K) mod p for each of np primes p < 2^62, by NW-Ryser in Montgomery
 * arithmetic.  kmod is [np][n*n] (row-major K reduced mod primes[q]).
 * out[q] = perm(K) mod primes[q]. */
void orc_perm_mod_primes(const uint64_t* kmod, int n, const uint64_t* primes, int np,
                         int threads, uint64_t* out);

/* Same for a Gaussian-integer matrix K = Kre + i*Kim (both [np][n*n] mod p).
 * out_re[q] + i*out_im[q] = perm(K) mod primes[q]. */
void orc_perm_mod_primes_gauss(const uint64_t* kre, const uint64_t* kim, int n,
                               const uint64_t* primes, int np, int threads,
                               uint64_t* out_re, uint64_t* out_im);

#ifdef __cplusplus
}
#endif

#endif
