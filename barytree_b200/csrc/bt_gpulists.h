// bt_gpulists.h -- MAC interaction lists traversed on the GPU (internal).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

#include "bt_host.h"

namespace bt {

// Particle-cluster (and cluster-particle) lists on the device: for every leaf
// of `bat` (a batch), a depth-first traversal of `trav` from the root of the
// batch's system with the reference's comparisons in FP64 (no contraction),
// so membership and order equal the host traversal's (bt_plan_traverse).
// ap/pp receive host CSR arrays (rows = bat->nleaves).  `work` is device
// memory of `work_bytes`.  Returns 0, a cudaError_t, or -1 when the traversal
// does not fit (too deep for the shared-memory stacks, or the work memory too
// small for the entries) -- the caller then traverses on the host.
int gpu_pc_lists(const bt_tree *trav, const bt_tree *bat, const bt_params *o, void *work, size_t work_bytes,
                 bt_csr *ap, bt_csr *pp, cudaStream_t st, long long *launches);

}  // namespace bt
