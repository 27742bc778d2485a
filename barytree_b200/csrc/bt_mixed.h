// bt_mixed.h -- launchers of the mixed-precision kernels (internal).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace bt {

constexpr int MX_MAX_DEG = 12;

// Near-field pairs closer than this fraction of the two leaves' summed radii
// are evaluated in FP64 (the rest of the mixed near field is FP32).
#ifndef BT_CLOSE_FRAC
#define BT_CLOSE_FRAC 0.01
#endif
constexpr double MX_CLOSE_FRAC = BT_CLOSE_FRAC;

// Tile shapes of the particle-output kernel (chosen by the autotuner): a
// work item is MX_CHUNK targets of one target leaf, evaluated by
// MX_CHUNK / tpt threads with tpt targets each; the near field streams
// source leaves through shared memory in tiles of `tile` particles.
constexpr int MX_CHUNK = 256;
constexpr int MX_TILE_MAX = 2048;
inline bool mixed_shape_valid(int tpt, int tile)
{
    return (tpt == 1 || tpt == 2 || tpt == 4) && (tile == 512 || tile == 1024 || tile == MX_TILE_MAX);
}

struct MixedTargetsArgs {
    int n, max_np1, nitems;
    const int2 *items;
    int *queue;                                 // work-queue counter (zeroed), or nullptr: one block per item
    bool herm;                                  // Hermite far field (Q32: 8 moments of P per node)
    const int *leaf_node, *t_ibeg, *t_numpar;
    const double *t_ctr;                        // target node centres (FP64, 3 per node)
    const float4 *tpos;                         // targets relative to their leaf centre
    const int64_t *a_off; const int *a_idx;     // source clusters per target leaf
    const unsigned char *a_deg;                 // per-entry degree (nullptr: all n)
    const double *s_grid[MX_MAX_DEG + 1];       // per degree: node grids (FP64)
    const float *Q32[MX_MAX_DEG + 1];           // per degree: proxy charges (FP32)
    const int64_t *d_off; const int *d_idx;     // source leaves per target leaf
    const unsigned char *d_flag;                // 1: leaf boxes within the close-pair distance
    const int *s_ibeg, *s_numpar;
    const double *s_ctr;                        // source node centres
    const float4 *spos;                         // sources relative to their leaf centre, with charge
    const double *t_rad, *s_rad;                // node radii (close-pair threshold)
    const double *tx64, *ty64, *tz64;           // FP64 coordinates and charges for close pairs
    const double *sx64, *sy64, *sz64, *sq64;
    double kc;                                  // mixed_kernel_constant()
    double kp;                                  // kernel parameter (FP64 close pairs)
    double *pot;
    int tpt, tile;                              // targets per thread, near-field source tile
};

struct MixedGridsArgs {
    int n, nitems;
    const int2 *items;
    int *queue;                                 // work-queue counter (zeroed), or nullptr: one block per item
    const double *t_grid, *t_ctr;
    const int64_t *c_off; const int *c_idx;     // M2L source clusters per target node
    const int64_t *p_off; const int *p_idx;     // CP source leaves per target node
    const int *s_ibeg, *s_numpar;
    const double *s_grid, *s_ctr;
    const float *Q32;
    const float4 *spos;
    double kc;                                  // mixed_kernel_constant()
    double *Phi;
};

void launch_rel_positions(int nleaves, const int *leaves, const int *ibeg, const int *numpar, const double *ctr,
                          const double *x, const double *y, const double *z, const double *q, float4 *out,
                          cudaStream_t st);
void launch_to_f32(size_t n, const double *src, float *dst, cudaStream_t st);
void launch_eval_targets_mixed(int kernel, const MixedTargetsArgs &a, cudaStream_t st);
void launch_eval_grids_mixed(int kernel, const MixedGridsArgs &a, cudaStream_t st);
int mixed_targets_chunk();                                   // targets per work item
double mixed_kernel_constant(int kernel, double kernel_param);

}  // namespace bt
