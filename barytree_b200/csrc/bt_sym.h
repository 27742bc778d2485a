// bt_sym.h -- symmetric near-field pairs of the mixed path (internal).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace bt {

// Largest leaf the symmetric pass takes (particles).
constexpr int SYM_MAX_LEAF = 2048;

struct SymArgs {
    int npairs;
    const int2 *pair;             // (A, B) leaf nodes, A != B
    const int64_t *slot;          // per pair: A side at slot[p], B side at slot[p] + numpar[A]
    const int *ibeg, *numpar;     // per node (the target tree is the source tree)
    const double *ctr;            // node centres, 3 per node
    const float4 *pos;            // particles relative to their leaf centre, with charge
    float *partial;               // per pair, per particle of A then of B: the pair's potential there
    float kc;                     // mixed_kernel_constant()
    // pairs of leaves within the close-pair distance of each other (launch_pp_sym_close)
    const double *rad;            // node radii
    const double *box;            // node boxes, x0 x1 y0 y1 z0 z1 per node
    const double *x64, *y64, *z64, *q64;   // FP64 particles in tree order
    double kp;                    // kernel parameter (FP64 close pairs)
};

struct SymGatherArgs {
    int nleaves;
    const int *leaf_node;
    const int *ibeg, *numpar;
    const int64_t *in_off;        // per unit: partial vectors addressed to it, in pair order
    const int64_t *in_slot;
    const float *partial;
    double *pot;                  // += the sum of the partial vectors, FP64, in that order
};

// Pairs whose leaf boxes are farther apart than the close-pair distance.
void launch_pp_sym(int kernel, const SymArgs &a, cudaStream_t st);
// Pairs whose boxes lie within it: FP32 distances below the close-pair
// distance are clamped to it, and each clamped pair's two terms are replaced
// by FP64 ones (from the FP64 particles) before the slices are written.
void launch_pp_sym_close(int kernel, const SymArgs &a, cudaStream_t st);
void launch_sym_gather(const SymGatherArgs &a, cudaStream_t st);

}  // namespace bt
