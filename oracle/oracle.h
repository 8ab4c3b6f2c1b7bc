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

/* Sequential importance sampling estimate of the number of perfect matchings
 * of a 0/1 pattern, restating aspSingleGPU / rasmussenScaleAB
 * (Algorithms/GPU/Sparse/aspSingleGPU.cuh:45-165,
 * Algorithms/GPU/Sparse/ApproximateSparseKernelDefinitions.cuh:32-290): host
 * scaling (50 alternating column/row passes), then per sample and per row in
 * order 10 scaling passes over the row's columns and the row, a draw with
 * probability rv_i*cv_j, and degree-1 propagation from the removed column
 * and row.  Pattern in both orientations (rptr/col, cptr/row, indices
 * ascending, no duplicates).  Sample k draws from SplitMix64 seeded with
 * seed ^ (k * 0xD1B54A32D192ED03).  Float arithmetic without contraction,
 * in the same order as the product, so estimates match it bit for bit.
 * orc_rasmussen_init fills rv[n], cv[n]; orc_rasmussen_samples writes the
 * estimates of samples first .. first+count-1. */
void orc_rasmussen_init(int n, const int* rptr, const int* col, const int* cptr, const int* row,
                        float* rv, float* cv);
void orc_rasmussen_samples(int n, const int* rptr, const int* col, const int* cptr, const int* row,
                           const float* rv0, const float* cv0, uint64_t seed, uint64_t first,
                           uint64_t count, int threads, double* out);

#ifdef __cplusplus
}
#endif

#endif
