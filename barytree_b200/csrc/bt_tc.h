// bt_tc.h -- tensor-core (tcgen05) kernels of barytree_b200 (internal).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace bt {

// A chunk of a node's particles for the Hermite P2M (the same as HermChunk of
// bt_device.h): slot < 0 writes the node's moments, else partial slot `slot`.
struct HermChunkTc {
    int node, begin, count, slot;
};

// Leaf P2M (Lagrange) on the tensor cores in 3xTF32 with FP32 accumulation,
// for degrees with n + 1 <= 16 ((n+1)^2 rows in one or two 128-row tiles).  Same output layout as launch_p2m
// (Q[node * P + k1 + (n+1) (k2 + (n+1) k3)], FP64).  *err is set to 1 if a
// bounded wait for the tensor core expired (the leaf's Q is then not written).
bool p2m_tc_supported(int n);
void launch_p2m_tc(int n, int nleaves, const int *leaves, const int *ibeg, const int *numpar, const double *grid,
                   const double *sx, const double *sy, const double *sz, const double *sq, double *Q, int *err,
                   cudaStream_t st);

bool l2p_tc_supported(int n);     // n + 1 <= 11: the (n+1)^2 columns in one N = 128 MMA
// L2P (Lagrange) at the target leaves on the tensor cores: each item (leaf,
// chunk of 128 targets) adds its targets' interpolated grid values to pot
// (3xTF32, FP32 accumulation); same items and layout as launch_l2p, degrees
// with (n+1)^2 <= 128.  *err as for launch_p2m_tc.
void launch_l2p_tc(int n, int nitems, const int2 *items, const int *leaf_node, const int *t_ibeg,
                   const int *t_numpar, const double *t_grid, const double *Phi, const double *tx, const double *ty,
                   const double *tz, double *pot, int *err, cudaStream_t st);

// Hermite P2M on the tensor cores for degrees with n + 1 <= 8: the 8
// moments of every chunk's node (or its partial slot), as launch_p2m_hermite
// writes them before its reduction; *err as for launch_p2m_tc.
bool p2m_hermite_tc_supported(int n);
void launch_p2m_hermite_tc(int n, int nchunks, const HermChunkTc *chunks, const double *grid, const double *box_len,
                           const double *ww, const double *sx, const double *sy, const double *sz, const double *sq,
                           double *Q, double *partial, int *err, cudaStream_t st);

// Inference of the degree selector's MLP (weights as bt_learned.h lays them
// out, B rows of 6 features -> 11 outputs) on the tensor cores, 3xTF32 with
// FP32 accumulation; *err as for launch_p2m_tc.
void mlp_infer_tc(const float *w, int64_t B, const float *X, float *Y, int *err, cudaStream_t st);

}  // namespace bt
