/*
 * superman_b200 — C ABI of the B200 (sm_100a) matrix-permanent library.
 *
 * This is the drop-in boundary for SUPerman's Ryser/Gray-code hot path.  Each
 * entry point replaces one reference interface (cited per declaration, paths
 * relative to the SUPerman source tree).  Plain pointers and sizes only; every
 * call returns a status code instead of exiting (the reference's gpuErrchk
 * calls exit(), Algorithms/GPU/GPUHelpers.cuh:77-85).
 *
 * Matrices are row-major, n x n, 1 <= n <= 63 (the reference's limit,
 * CommonFiles/DecomposePerman.h:185-188 and Algorithms/GPU/GPUHelpers.cuh:38).
 * Inputs are caller-owned host arrays unless the name ends in _dev.
 */
#ifndef SUPERMAN_B200_H
#define SUPERMAN_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SPB_API __attribute__((visibility("default")))
#else
#define SPB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status ---- */
enum spb_status {
    SPB_OK = 0,
    SPB_ERR_INVALID = 1,    /* bad argument: null pointer, n out of range      */
    SPB_ERR_CUDA = 2,       /* a CUDA runtime call failed (see spb_last_error) */
    SPB_ERR_NO_DEVICE = 3,  /* no usable CUDA device                           */
    SPB_ERR_OOM = 4,        /* device or host allocation failed                */
    SPB_ERR_OVERFLOW = 5,   /* exact integer result does not fit               */
    SPB_ERR_TIMEOUT = 6,    /* a bounded wait ran out                          */
    SPB_ERR_CANCELLED = 7,  /* the request was cancelled                       */
    SPB_ERR_BUSY = 8,       /* admission refused: queue or scratch full        */
    SPB_ERR_IO = 9,         /* file could not be opened or parsed              */
    SPB_ERR_NOT_SQUARE = 10,/* matrix file header is not square                */
    SPB_ERR_ACCURACY = 11   /* SPB_PREC_FP32: the result (returned) has an
                               estimated relative error above rel_tol          */
};

/* Precision modes.  SPB_PREC_FP64 corresponds to the reference's default
 * `calculation_precision=kahan` (CommonFiles/Settings.h:59-65, IO/IO.h:178)
 * and SPB_PREC_DD to `calculation_precision=dd`. */
enum spb_precision {
    SPB_PREC_FP64 = 0, /* FP64 row sums and products, double-double sum      */
    SPB_PREC_DD = 1,   /* + double-double re-evaluation of dominant units    */
    SPB_PREC_FP32 = 2  /* FP32 row sums and products (double-double unit
                          bases and sum), 3 <= n <= 40: faster, relative
                          error of order kappa * n * 2^-24.  The call
                          estimates that error (out->err_est, from the sum
                          of squared terms) and returns SPB_ERR_ACCURACY,
                          with the result filled in, when it exceeds
                          rel_tol (0 = 1e-12, which FP32 products never
                          meet: pass the bound the caller accepts)        */
};

/* Walk used by spb_perm_sparse_f64. */
enum spb_sparse_walk {
    SPB_SPARSE_WALK_AUTO = 0,   /* row-compacted walk when its cost model wins   */
    SPB_SPARSE_WALK_NEVER = 1,  /* always the dense walk                         */
    SPB_SPARSE_WALK_ALWAYS = 2  /* row-compacted walk whenever the pattern allows */
};

typedef struct spb_options {
    int device;            /* CUDA ordinal (Settings::deviceID)              */
    int precision;         /* enum spb_precision                             */
    double rel_tol;        /* SPB_PREC_DD target relative error (0 = 1e-13);
                              SPB_PREC_FP32 accepted error (0 = 1e-12)      */
    int unit_bits;         /* log2 Gray terms per unit; 0 = automatic.  A
                              width whose tables do not fit shared memory
                              (the walk's, or with SPB_PREC_DD both words
                              of the refinement's) is refused with
                              SPB_ERR_INVALID before any launch             */
    int threads_per_block; /* 0 = automatic                                  */
    int blocks;            /* 0 = automatic (persistent: one CTA per SM)     */
    void* stream;          /* cudaStream_t to run on; NULL = library stream  */
    int sparse_walk;       /* enum spb_sparse_walk (spb_perm_sparse_f64)     */
    int replay_listing;    /* SPB_PREC_DD: 1 = list the units to refine by
                              replaying the walk (its own unit bases) instead
                              of the first pass's list or the parallel scan;
                              same result, slower (for verification)        */
    int small_call;        /* >= 0: real matrices with 4 <= n <= 26 run as one
                              fused kernel (tables, walk, threshold and
                              refinement); < 0: as separate kernels        */
    int skip_timing;       /* 1: the dense entry points skip their device
                              timing (no elapsed-time queries; the replayed
                              fused call records no events); kernel_s and
                              device_s in spb_result are then 0.  About 6 us
                              less per call, for callers that time calls
                              themselves                                    */
} spb_options;

typedef struct spb_result {
    double value;          /* permanent (real part), rounded double-double  */
    double value_lo;       /* low word of the double-double result          */
    double imag;           /* imaginary part (complex entry points)         */
    double imag_lo;
    double elapsed_s;      /* wall time of the whole call                   */
    double kernel_s;       /* device time of the Gray-walk kernels          */
    double device_s;       /* device time of the whole call on its stream:
                              input copy (if any), kernels, result copy     */
    double err_est;        /* estimated relative error (statistical); for
                              spb_perm_approx the relative standard error */
    uint64_t gray_steps;   /* Gray steps walked, n*2^(n-1) (every walk is
                              Nijenhuis-Wilf); spb_perm_approx: samples    */
    uint64_t refined_units;/* units re-evaluated in double-double           */
    int status;            /* enum spb_status                               */
    int launches;          /* kernels launched by the call                  */
    int active_rows;       /* rows varying inside a Gray unit: n for the
                              dense walk, fewer for the row-compacted walk  */
} spb_result;

/* Fills *opt with the defaults (device 0, SPB_PREC_FP64, automatic shape). */
SPB_API void spb_default_options(spb_options* opt);

/* Message of the last failed call on this host thread ("" if none). */
SPB_API const char* spb_last_error(void);

/* Static name of a status code. */
SPB_API const char* spb_status_string(int status);

/* Library version as major*10000 + minor*100 + patch. */
SPB_API int spb_version(void);

/* Number of CUDA devices visible (0 when none; never fails). */
SPB_API int spb_device_count(void);

/* Dense real permanent by the Nijenhuis–Wilf Ryser formula with Gray-code
 * enumeration.  Replaces the dense single-GPU driver
 * dpSingleGPU<C,S,Algo,Shared>::permanentFunction
 * (Algorithms/GPU/Dense/dpSingleGPU.cuh:45-219) and its kernels
 * xRegisterMShared[Kahan] (Algorithms/GPU/Dense/DenseKernelDefinitions.cuh:
 * 189-264, 331-405).  a: n*n doubles, row-major.  A matrix with zeros may
 * run on the row-compacted walk of spb_perm_sparse_f64 when its cost model
 * wins (opt->sparse_walk; out->active_rows < n then). */
SPB_API int spb_perm_dense_f64(const double* a, int n, const spb_options* opt, spb_result* out);

/* Sparse real permanent from compressed-column arrays, the layout of the
 * reference's SparseMatrix (Structures/SparseMatrix.h:61-101): column c holds
 * rows[cptrs[c] .. cptrs[c+1]-1] with values cvals[...]; nnz = cptrs[n];
 * duplicate entries are summed.  Replaces spSingleGPU<C,S,Algo>::
 * permanentFunction (Algorithms/GPU/Sparse/spSingleGPU.cuh:45-234) with its
 * kernels (Algorithms/GPU/Sparse/SparseKernelDefinitions.cuh:33-509), and the
 * per-matrix generated kernels (Algorithms/GPU/CodeGeneration/
 * KernelGenerator.cuh:114-176): rows and columns are permuted so that the
 * rows varying inside a Gray unit are few, and a walk compiled for that row
 * count runs (opt->sparse_walk; out->active_rows reports it). */
SPB_API int spb_perm_sparse_f64(const int* cptrs, const int* rows, const double* cvals, int n,
                                const spb_options* opt, spb_result* out);

/* The plan spb_perm_sparse_f64 would run for a row-major n x n matrix under
 * sparse_walk `mode`, without running it: *na active rows (n = the dense
 * walk), *w low columns, and the row and column orders (new position ->
 * original index; either may be NULL).  In the permuted matrix rows
 * na..n-1 are zero in columns 0..w-1.  CPU only. */
SPB_API int spb_sparse_plan(const double* a, int n, int mode, int* na, int* w, int* row_order, int* col_order);

/* Monte-Carlo estimate of the permanent of the nonzero pattern of an n x n
 * matrix (its number of perfect matchings; the values are not used), for
 * any n up to 2^20 — beyond the exact paths' n <= 63.  Replaces aspSingleGPU
 * (Algorithms/GPU/Sparse/aspSingleGPU.cuh:45-165) with its kernel
 * rasmussenScaleAB (Algorithms/GPU/Sparse/ApproximateSparseKernelDefinitions.cuh:
 * 177-290): sequential importance sampling over the rows in order, with the
 * same host scaling (50 passes), per-row scaling (10 passes) and degree-1
 * propagation.  The pattern comes as compressed-column arrays (cptrs[n+1],
 * rows[cptrs[n]]).  `samples` estimates are averaged; sample k draws from its
 * own stream of `seed`, so the result does not depend on the launch shape.
 * out->value is the mean, out->err_est the standard error relative to it,
 * out->gray_steps the number of samples. */
SPB_API int spb_perm_approx(const int* cptrs, const int* rows, int n, uint64_t samples, uint64_t seed,
                            const spb_options* opt, spb_result* out);

/* The individual estimates of samples first .. first+count-1 of
 * spb_perm_approx (same pattern, same seed), into estimates[count] (host). */
SPB_API int spb_approx_samples(const int* cptrs, const int* rows, int n, uint64_t first, uint64_t count,
                               uint64_t seed, double* estimates);

/* Same on a device-resident row-major matrix. */
SPB_API int spb_perm_dense_f64_dev(const double* d_a, int n, const spb_options* opt,
                           spb_result* out);

/* Dense complex128 permanent.  Replaces gpuComputeComplex
 * (Algorithms/Complex/gpuComputeComplex.cu:199-418, declared in
 * Algorithms/Complex/gpuComputeComplex.cuh:33) and its kernel
 * xRegisterMSharedComplex (gpuComputeComplex.cu:39-117).
 * a: n*n (re, im) pairs, row-major, 2*n*n doubles. */
SPB_API int spb_perm_dense_c128(const double* a, int n, const spb_options* opt, spb_result* out);

/* Same on a device-resident interleaved matrix. */
SPB_API int spb_perm_dense_c128_dev(const double* d_a, int n, const spb_options* opt,
                            spb_result* out);

/* Permanents of `count` n x n matrices in one launch, one warp per matrix
 * (1 <= n <= 24).  d_mats: device, count consecutive row-major matrices
 * (is_complex: interleaved re/im, 2*n*n doubles each); d_out: device,
 * 2 doubles per component per matrix, the permanent as a double-double
 * (hi, lo).  Asynchronous on `stream` (NULL = default stream); allocates
 * nothing.  Batched counterpart of the dense drivers above for the many
 * small permanents a serving queue or a decomposition produces; the
 * reference runs each of them through its own chunk loop and launches
 * (Algorithms/GPU/Dense/dpSingleGPU.cuh:156-199). */
SPB_API int spb_perm_batch_dev(const double* d_mats, int n, int is_complex, int count,
                               double* d_out, void* stream);

/* Exact permanent of a 0/1 matrix (a: n*n bytes, row-major, nonzero = 1) by
 * plain Ryser over all 2^n column subsets in wrap-around integer arithmetic
 * whose width (128, 192 or 320 bits) is chosen from a Bregman-Minc bound, so
 * the result is exact for every n <= 63.  limbs receives the permanent as a
 * 320-bit two's-complement integer in ten little-endian 32-bit words;
 * out->value is its nearest double.  Replaces the reference's 0/1 handling,
 * which reads the pattern (IO/IO.h:441-443) and runs the FP64 dense path
 * (Algorithms/GPU/Dense/dpSingleGPU.cuh:45-219), inexact beyond 2^53. */
SPB_API int spb_perm_binary(const uint8_t* a, int n, const spb_options* opt, uint32_t* limbs,
                            spb_result* out);

/* Dense real permanent that allocates nothing, for callers that cannot let a
 * library call cudaMalloc/cudaFree: programs that reserve all device memory
 * for their own pool allocator, and latency-bound request loops that cannot
 * take cudaFree's device-wide synchronisation or an allocation failure
 * mid-request.  d_a: device, n*n doubles row-major; d_out: device, 2 doubles
 * receiving the permanent as (hi, lo).  Runs asynchronously on `stream`
 * (NULL = the default stream); read d_out after synchronising.
 * Precision is that of SPB_PREC_FP64 (FP64 row sums and products,
 * double-double sums, no double-double refinement): about 1e-13 relative at
 * n=24 and 3e-12 at n=32 on U[0,1) entries, so lo is not a double-double
 * accurate correction.  Working memory is one fixed 256 KiB device array per
 * GPU inside the library, so n is limited to 1..40 (larger n:
 * SPB_ERR_INVALID).  The first call on a device looks up that array's address
 * and loads the kernels the call can launch (CUDA loads modules lazily by
 * default, which can allocate): make it before reserving the rest of device
 * memory for a pool, and before any stream capture.  All calls share the
 * array: calls that overlap on the GPU race.
 * No counterpart in the reference, which allocates on every call
 * (Algorithms/GPU/Dense/dpSingleGPU.cuh:138-144). */
SPB_API int spb_perm_dense_f64_noalloc(const double* d_a, int n, double* d_out, void* stream);

/* ------------------------------------------------ host pipeline ---- */

/* Outcome of the reference's top-level flow (main.cpp:42-151). */
typedef struct spb_pipeline_result {
    double permanent;  /* real permanent, or the real part                   */
    double imag;       /* imaginary part (complex=true)                      */
    double time_s;     /* the reference's "Computed in" time                 */
    double avg_n;      /* mean size of the decomposed pieces ("Average N")   */
    double avg_nnz;    /* mean nonzeros of the pieces ("Average NNZ")        */
    int components;    /* bipartite connected components after pruning       */
    int pieces;        /* pieces computed ("Submatrix count")                */
    int algorithm;     /* Algorithm enum value chosen (Settings.h)           */
    int status;
} spb_pipeline_result;

/* Runs main.cpp's real-matrix flow on an in-memory row-major matrix:
 * perfect-matching pruning (IO/IO.h:477-508, IO/dm.cpp:441-501), connected
 * components (IO/dm.h:43-107), AlgorithmSelector (CommonFiles/
 * AlgorithmSelector.h:49-141), DecomposePerman (CommonFiles/
 * DecomposePerman.h:76-557) and the GPU drivers, with settings given as the
 * reference's key=value arguments (IO/IO.h:163-401), e.g. "algorithm=auto",
 * "calculation_precision=dd", "binary=true", "scaling=true".  mode=cpu and
 * the multi-GPU modes are reported as unavailable (SPB_ERR_INVALID). */
SPB_API int spb_perm_pipeline(const double* a, int n, const char* const* args, int nargs,
                              spb_pipeline_result* out);

/* The whole reference program on a matrix file: args as on its command line
 * ("filename=...", "complex=true", "binary=true", "undirected=true", ...);
 * replaces main.cpp:42-151 with IO::readMatrix / IO::readComplex
 * (IO/IO.h:403-596). */
SPB_API int spb_perm_file(const char* const* args, int nargs, spb_pipeline_result* out);

/* Reads a matrix file as IO::readMatrix / IO::readComplex do (IO/IO.h:403-596),
 * pruning included for real matrices.  *n is always set; the entries are
 * copied to `out` (row-major; interleaved re/im when is_complex) when out is
 * non-null and n <= max_n.  CPU only. */
SPB_API int spb_read_matrix(const char* path, int binary, int undirected, int is_complex, double* out,
                            int max_n, int* n, double* sparsity);

/* Perfect-matching pruning of a dense row-major matrix into out (n*n); sets
 * *has_perfect_matching (0: the permanent is structurally zero and out is
 * all zeros).  Replaces dm() (IO/dm.cpp:441-501).  CPU only. */
SPB_API int spb_dm_prune(const double* a, int n, double* out, int* has_perfect_matching);

/* The pieces main.cpp's real-matrix flow (main.cpp:63-110) computes for a
 * matrix, without computing them: perfect-matching pruning (IO/IO.h:477-508),
 * connected components (IO/dm.h:43-107) and DecomposePerman
 * (CommonFiles/DecomposePerman.h:76-557) on each component, with the default
 * settings.  The permanent of the matrix is the product over the
 * *components of the sum of the permanents of each component's pieces (a
 * component without pieces contributes 0: a structurally zero permanent is
 * one component with no pieces).  *count pieces; sizes[k], piece_component[k]
 * and the row-major entries concatenated in data.  Pass sizes =
 * piece_component = data = NULL to query *components and *count alone.
 * The reference prints the piece count and their mean size as "Submatrix
 * count" and "Average N" (main.cpp:117-121).  CPU only. */
SPB_API int spb_plan_pieces(const double* a, int n, int* components, int* count, int* sizes,
                            int* piece_component, double* data, int max_pieces, size_t max_doubles);

/* The reference's row/column orderings (IO/IO.h:598-1112) applied to a
 * row-major n x n matrix: order is "colSort", "rowSort" (param 0 ascending,
 * else descending), "skipOrder", "UTOrder", "colIndexMinimizationOrder",
 * "alphaOrder" (param = alpha, 0 means 2) or "randomOrder" (param = seed,
 * 0 random).  The permanent is unchanged.  CPU only. */
SPB_API int spb_reorder(const double* a, int n, const char* order, unsigned long long param, double* out);

/* The pieces DecomposePerman (CommonFiles/DecomposePerman.h:120-198) would
 * compute for a matrix, without computing them: *count pieces, sizes[k] and
 * their row-major entries concatenated in data.  Pass sizes = data = NULL to
 * query *count alone.  The permanents of the pieces sum to the permanent of
 * the matrix.  CPU only. */
SPB_API int spb_decompose(const double* a, int n, int* count, int* sizes, double* data, int max_pieces,
                          size_t max_doubles);

/* ------------------------------------------------------- serving ---- */
/* A request loop for many permanents of mixed sizes (no counterpart in the
 * reference, which computes one matrix per process run; the per-request
 * semantics are those of the single-GPU drivers,
 * Algorithms/GPU/Dense/dpSingleGPU.cuh:156-209).  A request is admitted
 * while its matrix fits the server's device pool (admit_bytes of device
 * memory, reserved from admission to completion); a real matrix with zero
 * entries is pruned and decomposed on the host as the reference's main flow
 * does (spb_plan_pieces), and its pieces run as independent requests.
 * Small matrices (n <= 20) are packed per (n, real/complex) into batched
 * launches (one warp per matrix; a batch shape used a few times is captured
 * once in a CUDA graph and replayed); mid-size ones (21 <= n <= batch_max_n)
 * are batched when enough of one shape are queued and otherwise run like the
 * large ones; large ones run the whole-GPU walk on large_workers streams with
 * their own working memory, so batches and whole-GPU calls overlap on the
 * device.  A request's result does not depend on what it was batched with. */
typedef struct spb_server_config {
    int device;
    int batch_max_n;      /* n <= this may go through batched launches (1..24; 0 = 24) */
    int max_batch;        /* matrices per batched launch (0 = 2048)                     */
    int slots;            /* batched launches in flight (0 = 4)                         */
    double max_wait_s;    /* longest a small request waits for its batch to fill       */
    size_t admit_bytes;   /* device pool for admitted matrices (0 = 256 MiB)            */
    int precision;        /* enum spb_precision of whole-GPU requests (a zero-filled
                             config gives SPB_PREC_FP64; spb_server_default_config and
                             a NULL config give SPB_PREC_DD)                             */
    int use_graphs;       /* >= 0: replay captured batch shapes (default); < 0: plain launches */
    int large_workers;    /* concurrent whole-GPU calls (0 = 2)                         */
    int split;            /* >= 0: decompose real matrices with zeros (default); < 0: off */
} spb_server_config;

typedef struct spb_request_result {
    double re, re_lo, im, im_lo; /* the permanent (double-double per component) */
    double submit_s, done_s;     /* steady-clock seconds: admission, completion */
    int n, is_complex;
    int status;                  /* SPB_OK, SPB_ERR_CANCELLED or a failure       */
} spb_request_result;

typedef struct spb_server_stats {
    uint64_t submitted, completed, rejected, cancelled;
    uint64_t batches, batched_requests, graph_launches, graphs_captured, large_launches;
    size_t queued_bytes;          /* device pool bytes reserved by requests in the server */
    uint64_t split_requests;      /* requests decomposed into pieces                       */
    uint64_t pieces;              /* pieces they produced                                  */
    uint64_t mid_to_large;        /* mid-size requests run as whole-GPU calls               */
    size_t pool_bytes;            /* device pool size                                      */
} spb_server_stats;

/* Fills *cfg with the defaults (device 0, batch_max_n 24, 2048 per batch,
 * 4 slots, 200 us fill window, 256 MiB pool, SPB_PREC_DD, graphs on, 2
 * whole-GPU workers, decomposition on). */
SPB_API void spb_server_default_config(spb_server_config* cfg);
SPB_API int spb_server_create(const spb_server_config* cfg, void** server);
/* Copies the row-major matrix (interleaved re/im when is_complex) into the
 * server's pool; SPB_ERR_BUSY when admission refuses it (the pool is full). */
SPB_API int spb_server_submit(void* server, const double* a, int n, int is_complex, uint64_t* ticket);
/* Submits `count` matrices in one call (sizes ns[k], flags is_complex[k],
 * entries concatenated row-major in `mats`); tickets[k] receives each ticket,
 * or 0 where admission refused the matrix.  Returns the number admitted in
 * *admitted.  For clients that receive requests in bulk. */
SPB_API int spb_server_submit_many(void* server, const double* mats, const int* ns, const int* is_complex,
                                   int count, uint64_t* tickets, int* admitted);
/* SPB_OK and the result when done (the ticket is then released), SPB_ERR_BUSY
 * while pending, SPB_ERR_INVALID for an unknown ticket. */
SPB_API int spb_server_poll(void* server, uint64_t ticket, spb_request_result* out);
/* Like poll but waits up to timeout_s; SPB_ERR_TIMEOUT if still pending. */
SPB_API int spb_server_wait(void* server, uint64_t ticket, double timeout_s, spb_request_result* out);
/* Cancels a queued request (SPB_OK); an in-flight one completes as cancelled. */
SPB_API int spb_server_cancel(void* server, uint64_t ticket);
SPB_API int spb_server_get_stats(void* server, spb_server_stats* out);
/* Stops the workers after the work in flight and frees the server. */
SPB_API int spb_server_destroy(void* server);
/* Steady-clock seconds on the clock the request timestamps use. */
SPB_API double spb_now(void);

/* Fault injection for tests: each of the next `count` library allocations
 * (device scratch, refinement list, pinned staging, serving slots) fails with
 * SPB_ERR_OOM without allocating; the calls after them work normally.  0
 * clears it.  Host-side only: no GPU fault is involved. */
SPB_API void spb_debug_fail_allocations(int count);

/* Measured pipe throughput used as the roofline denominator: which = 0 gives
 * FP64 FMA thread-instructions per second, which = 1 gives int32 multiply-add
 * thread-instructions per second (best of three timed launches).  No
 * reference counterpart: the reference reports no roofline. */
SPB_API int spb_measure_pipe_peak(int device, int which, double* ops_per_s);

#ifdef __cplusplus
}
#endif

#endif /* SUPERMAN_B200_H */
