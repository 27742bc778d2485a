// bt_learned.h -- learned degree selection (internal).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace bt {

constexpr int MLP_IN = 6;
constexpr int MLP_H = 64;
constexpr int MLP_DMIN = 2, MLP_DMAX = 12;
constexpr int MLP_OUT = MLP_DMAX - MLP_DMIN + 1;       // log10 error at degrees 2..12
constexpr int MLP_PP = 255;                            // choice: evaluate directly
// weights: norm (mean[IN], std[IN]), W1[IN][H], b1[H], W2[H][H], b2, W3[H][H], b3, W4[H][OUT], b4[OUT]
constexpr int MLP_NWEIGHTS = 2 * MLP_IN + MLP_IN * MLP_H + MLP_H + 2 * (MLP_H * MLP_H + MLP_H) + MLP_H * MLP_OUT + MLP_OUT;
constexpr int LBL_TARGETS = 32;                        // targets sampled per labelled interaction

struct MlpView {
    float *norm;
    float *W[4];
    float *b[4];
};

struct FeatureArgs {
    int units;
    const int64_t *off; const int *idx;  // CSR of approx entries per target leaf unit
    const int *unit_node;                // unit -> target node
    const double *t_ctr, *s_ctr, *t_rad, *s_rad, *s_mom;
    const int *t_numpar, *s_numpar;
};

struct LabelArgs {
    const int *tnodes, *snodes;
    const int *t_ibeg, *t_numpar, *s_ibeg, *s_numpar;
    const double *tx, *ty, *tz, *sx, *sy, *sz, *sq;
    const double *t_ctr, *s_ctr, *s_mom;
    const double *grid[MLP_DMAX + 1];
    const double *Q[MLP_DMAX + 1];
    float *labels;
};

MlpView mlp_view(float *w);
void mlp_forward(const float *w, int B, const float *X, float *act, float *Yh, cudaStream_t st);
// Inference: mlp_infer_tc (bt_tc.h), on the tensor cores.
void mlp_forward_backward(const float *w, int B, const float *X, const float *Y, float *act, float *Yh, float *dbuf,
                          float *lossb, float *grad, cudaStream_t st);
void mlp_adam(int n, float *w, const float *g, float *m, float *v, float lr, int step, cudaStream_t st);
void gather_rows(int B, int width, const int *rows, const float *src, float *dst, cudaStream_t st);
// Source tree on the device for the node moments (lvl_off is a host array).
struct MomentTree {
    int nnodes, nleaves, max_depth;
    const int *leaves, *ibeg, *numpar, *nchild, *child, *lvl_nodes;
    const int *lvl_off;
};
// mom[2 i] = sum |q|, mom[2 i + 1] = sqrt(sum q^2) over node i's particles.
// Returns the number of kernel launches.
int launch_node_moments(const MomentTree &t, const double *q, double *mom, cudaStream_t st);
void launch_features(const FeatureArgs &a, int64_t nentries, float *out, cudaStream_t st);
void launch_features_pairs(const FeatureArgs &a, int n, const int *tnodes, const int *snodes, float *out,
                           cudaStream_t st);
void launch_labels(const LabelArgs &a, int nsamples, cudaStream_t st);
// Selection under one absolute error share per system (bt_learned.cu):
// sys_off = nsys + 1 offsets of each system's units (target leaves);
// unit_sums: 2 * units doubles, log_share: nsys floats of scratch.
void launch_select_share(const FeatureArgs &a, int nsys, const int *sys_off, const int *t_ibeg, const int64_t *d_off,
                         const int *d_idx, const int *s_ibeg, const double *sx, const double *sy, const double *sz,
                         const double *sq, const double *tx, const double *ty, const double *tz, double c_tol,
                         int64_t n, const float *pred, const float *feat, double *unit_sums, float *log_share,
                         unsigned char *choice, cudaStream_t st);

}  // namespace bt
