// Host-side entry of the dense driver (dense.cu), shared with the sparse
// entry point (sparse.cu).
#pragma once

#include "superman_b200.h"

namespace spb {
struct DeviceContext;
namespace dense {

// A row-compacted walk plan for a matrix already permuted by the caller:
// rows 0..na-1 are the rows with a nonzero in columns 0..w-1, rows na..n-1
// have none there (sparse_impl.cuh).
struct WalkPlan {
    int na;
    int w;
};

// One permanent on the GPU: the dense walk, or the row-compacted walk when
// plan is non-null with plan->na < n (real matrices on the host only).  ctx:
// the context whose stream and arenas the call uses (null: the device's
// shared context, opt->device).
int run(const double* a, bool a_on_device, int n, int comps, const spb_options* opt, spb_result* out,
        const WalkPlan* plan, DeviceContext* ctx = nullptr);

// A real matrix on the host: the row-compacted walk when opt->sparse_walk
// and the cost model pick it (sparse.cu), the dense walk otherwise.
int run_real_host(const double* a, int n, const spb_options* opt, spb_result* out,
                  DeviceContext* ctx = nullptr);

}  // namespace dense
}  // namespace spb
