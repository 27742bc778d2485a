// bt_gputree.h -- the tree build on the GPU (internal).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "bt_host.h"

namespace bt {

// Particles in tree order on the device; order[i] = caller index of sorted
// particle i.  q is null for targets.
struct GtArrays {
    double *x, *y, *z, *q;
    int *order;
};

// Device work memory gpu_build_tree / gpu_build_forest need besides `out`.
size_t gpu_tree_work_bytes(int n, int maxpar, bool with_q, int nsys = 1);

// Builds the tree of n particles (x, y, z, q: host or device memory; q may
// be null) with at most maxpar particles per leaf.  The sorted particles go
// to `out` (device arrays of n entries each, q only if q is given); the node
// arrays to *t.  Returns 0 or a cudaError_t.
int gpu_build_tree(int n, const double *x, const double *y, const double *z, const double *q, int maxpar,
                   GtArrays out, void *work, size_t work_bytes, bt_tree *t, cudaStream_t st, long long *launches);

// The same for nsys independent systems (system k: particles
// [sys_off[k], sys_off[k+1]) of the arrays): one forest, every system's nodes
// numbered consecutively in pre-order, particles sorted within their system.
int gpu_build_forest(int nsys, const int64_t *sys_off, const double *x, const double *y, const double *z,
                     const double *q, int maxpar, GtArrays out, void *work, size_t work_bytes, bt_tree *t,
                     cudaStream_t st, long long *launches);

// *equal = arrays a and b (device, n entries) hold the same bits; `flag` is
// 8 bytes of device scratch.  Returns 0 or a cudaError_t.
int gpu_arrays_equal(const double *a, const double *b, size_t n, unsigned long long *flag, bool *equal,
                     cudaStream_t st);

// Source line (bt_gputree.cu) of the last failing CUDA call of a build.
int gpu_tree_fail_line();

}  // namespace bt
