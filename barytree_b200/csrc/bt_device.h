// bt_device.h -- launchers of the barytree_b200 CUDA kernels (internal).
#pragma once

#include <cuda_runtime.h>

#include <vector>
#include <cstdint>

namespace bt {

struct EvalTargetsArgs {
    int n, nitems;
    const int2 *items;            // (target leaf unit, chunk), sorted by cost
    const int *leaf_node;         // unit -> target node
    const int *t_ibeg, *t_numpar;
    const int64_t *a_off; const int *a_idx;   // source clusters per unit
    const int64_t *d_off; const int *d_idx;   // source nodes per unit
    const int *s_ibeg, *s_numpar;
    const double *s_grid, *Q;
    const double *sx, *sy, *sz, *sq;
    const double *tx, *ty, *tz;
    double kp, kp2;                             // kernel_params[0], [1]
    double *pot;
    int tb = 1;                                 // targets per thread (1 or 2): items of tb * 128 targets
};

struct EvalGridsArgs {
    int n, nitems;
    const int2 *items;            // (target node, chunk of grid points)
    const double *t_grid;
    const int64_t *c_off; const int *c_idx;   // source clusters (M2L) per target node
    const int64_t *p_off; const int *p_idx;   // source nodes (CP) per target node
    const int *s_ibeg, *s_numpar;
    const double *s_grid, *Q;
    const double *sx, *sy, *sz, *sq;
    double kp, kp2;                             // kernel_params[0], [1]
    double *Phi;
};

void launch_p2m(int n, bool hermite, int nleaves, const int *leaves, int nnodes, const int *ibeg, const int *numpar,
                const double *grid, const double *box_len, const double *ww, const double *sx, const double *sy,
                const double *sz, const double *sq, double *Q, cudaStream_t st);
// Hermite P2M over particle chunks (see bt_device.cu).  slot < 0: the chunk
// is its node's only one and writes Q directly.
struct HermChunk {
    int node, begin, count, slot;
};
// Chunks of every node and, for nodes with several chunks, (node, first slot,
// slot count); returns the number of partial slots (8 (n+1)^3 doubles each).
int hermite_chunks(int nnodes, const int *ibeg, const int *numpar, std::vector<HermChunk> &chunks,
                   std::vector<int3> &red);
void launch_p2m_hermite(int n, int nchunks, const HermChunk *chunks, int nred, const int3 *red, const double *grid,
                        const double *box_len, const double *ww, const double *sx, const double *sy, const double *sz,
                        const double *sq, double *Q, double *partial, cudaStream_t st);
// Q of every node with several chunks: the sum of its partial moments in chunk order.
void launch_hermite_reduce(int n, int nred, const int3 *red, const double *partial, double *Q, cudaStream_t st);
void launch_m2m(int n, int nparents, const int *parents, const int *nchild, const int *child, const double *grid,
                double *Q, cudaStream_t st);
void launch_l2l(int n, int nparents, const int *parents, const int *nchild, const int *child, const double *grid,
                double *Phi, cudaStream_t st);
void launch_eval_targets(int kernel, bool hermite, const EvalTargetsArgs &a, cudaStream_t st);
// Targets per work item of launch_eval_targets with tb targets per thread, and
// the tb to use for target leaves with count[u] targets.
int fp64_targets_chunk(int tb);
int fp64_targets_per_thread(int nunits, const int *count);
void launch_eval_grids(int kernel, bool hermite, const EvalGridsArgs &a, cudaStream_t st);
void launch_l2p(int n, bool hermite, int nitems, const int2 *items, const int *leaf_node, const int *parent,
                const int *t_ibeg, const int *t_numpar, const double *t_grid, const double *box_len,
                const double *ww, const double *Phi, const double *tx, const double *ty, const double *tz,
                double *pot, cudaStream_t st, const double *mult = nullptr);
void launch_scatter(int n, const int *order, const double *src, double *dst, cudaStream_t st);
// dst[i] = src[order[i]] (inputs in caller order -> tree order)
void launch_gather(int n, const int *order, const double *src, double *dst, cudaStream_t st);
float run_probe(int which, int sms, double *ops, void *scratch, cudaStream_t st);
void launch_direct(int kernel, int nt, int ns, const double *tx, const double *ty, const double *tz,
                   const double *sx, const double *sy, const double *sz, const double *sq, double kp, double *out,
                   cudaStream_t st, double kp2 = 0.0);

}  // namespace bt
