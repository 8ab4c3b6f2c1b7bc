// Batched walk (batch.cu): one warp per matrix, n <= kMaxN.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace spb {
namespace batch {

constexpr int kMaxN = 24;
// Offsets in an offset table count units of kOffsetUnit doubles (256 bytes).
constexpr size_t kOffsetUnit = 32;

// Permanents of `count` matrices of n*n*(is_complex ? 2 : 1) doubles at
// dst + d_offs[m]*kOffsetUnit on the device, one warp per matrix; each warp
// first copies its matrix there from src + d_offs[m]*kOffsetUnit (page-locked
// host memory mapped into the device's address space, or device memory).
// Permanent m goes to d_out[m*2*comps ...] as for spb_perm_batch_dev.
// Asynchronous on s.
int launch_gathered(const double* src, double* dst, const unsigned* d_offs, int n, int is_complex, int count,
                    double* d_out, cudaStream_t s);

}  // namespace batch
}  // namespace spb
