// bt_ss.h -- launchers of the singularity-subtraction kernels (internal).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace bt {

struct SsTargetsArgs {
    int n, nitems;
    const int2 *items;                          // (target leaf unit, chunk of ss_chunk() targets)
    const int *leaf_node, *t_ibeg, *t_numpar;
    const int64_t *a_off; const int *a_idx;     // source clusters per unit
    const int64_t *d_off; const int *d_idx;     // source nodes per unit (direct)
    const int *s_ibeg, *s_numpar;
    const double *s_grid, *Q, *W;               // proxies of q*w and of w
    const double *sx, *sy, *sz, *sq, *sw;
    const double *tx, *ty, *tz, *tq;
    double kp, kp2;                             // kernel_params[0], [1]
    double *pot;
};

struct SsGridsArgs {
    int n, nitems;
    const int2 *items;
    const double *t_grid;
    const int64_t *c_off; const int *c_idx;     // M2L source clusters per target node
    const int64_t *p_off; const int *p_idx;     // CP source nodes per target node
    const int *s_ibeg, *s_numpar;
    const double *s_grid, *Q, *W;
    const double *sx, *sy, *sz, *sq, *sw;
    double kp;
    double *Phi_q, *Phi_w;
};

int ss_chunk();                                 // targets per work item of launch_ss_targets
void launch_ss_targets(int kernel, bool hermite, const SsTargetsArgs &a, cudaStream_t st);
void launch_ss_grids(int kernel, const SsGridsArgs &a, cudaStream_t st);
// Kernels with a singularity-subtraction direct sum (Coulomb, Yukawa and
// their regularized forms); the others ignore the singularity setting.
bool ss_direct_kernel(int kernel);
// out[t] = sum_j of the SS pair term over all sources (no correction term)
void launch_ss_direct(int kernel, int nt, int ns, const double *tx, const double *ty, const double *tz,
                      const double *tq, const double *sx, const double *sy, const double *sz, const double *sq,
                      const double *sw, double kp, double kp2, double *out, cudaStream_t st);
void launch_mul(int n, const double *a, const double *b, double *c, cudaStream_t st);
// pot[i] += c tq[i]
void launch_ss_correction(int n, double c, const double *tq, double *pot, cudaStream_t st);
// The same over work items (unit, chunk of `chunk` targets of the unit's leaf).
void launch_ss_correction_items(int nitems, const int2 *items, int chunk, const int *leaf_node, const int *ibeg,
                                const int *numpar, double c, const double *tq, double *pot, cudaStream_t st);
double ss_correction_constant(int kernel, double kp);

}  // namespace bt
