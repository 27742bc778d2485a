// bt_mixed.cu -- mixed-precision evaluation kernels of barytree_b200.
//
// Arithmetic: every kernel evaluation (PP, PC, CP, M2L) runs in FP32 on
// coordinates relative to the centre of the target leaf / node, so FP32 only
// ever sees displacements of the size of the interaction, never absolute
// positions.  Centre offsets between the two sides of an interaction are
// formed in FP64 and rounded once.  Per-interaction partial sums are FP32
// (far field: Kahan-compensated); they are folded into an FP64 per-target
// accumulator after every list entry / tile, which is the FP64 far+near
// reduction.  Tree boxes, Chebyshev node placement, exact-node coincidence
// tests and the barycentric passes stay FP64 (bt_device.cu).
//
// The far-field loops are instantiated per degree (NP1 = n+1, template) so
// the target-relative grid coordinates of one axis live in registers.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "bt_mixed.h"

namespace bt {

template <int KT>
__device__ __forceinline__ float kf_far(float r2, float q, float kp)
{
    if (KT == 1) {
        return q * rsqrtf(r2);
    } else if (KT == 2) {
        float rinv = rsqrtf(r2);
        float r = r2 * rinv;
        return q * rinv * __expf(-kp * r);
    } else {
        return q * rsqrtf(r2 + kp * kp);
    }
}

// PP: the reference skips r^2 <= DBL_MIN (Coulomb) / r <= DBL_MIN (Yukawa);
// in FP32 the coincident pair gives r2 == 0 exactly.
template <int KT>
__device__ __forceinline__ float kf_pp(float r2, float q, float kp)
{
    if (KT == 3) return q * rsqrtf(r2 + kp * kp);
    float v = kf_far<KT>(r2, q, kp);
    return r2 > 0.0f ? v : 0.0f;
}

__device__ __forceinline__ void kahan_add(float &s, float &c, float v)
{
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

constexpr int MX_THREADS = 128;
constexpr int MX_TILE = 1024;

// Far field of one source cluster at degree NP1-1 for one target at
// (x,y,z) relative to the target centre; g = grid coordinates relative to the
// same centre (FP32, smem), q = proxy charges (FP32, smem).
template <int KT, int NP1>
__device__ __forceinline__ float pc_cluster(float x, float y, float z, const float *g, const float *q, float kp)
{
    float gx[NP1];
#pragma unroll
    for (int k = 0; k < NP1; k++) gx[k] = x - g[k];
    float s = 0.f, c = 0.f;
    int j = 0;
    for (int k3 = 0; k3 < NP1; k3++) {
        float dz = z - g[2 * NP1 + k3];
        for (int k2 = 0; k2 < NP1; k2++) {
            float dy = y - g[NP1 + k2];
            float dyz = fmaf(dy, dy, dz * dz);
            float row = 0.f;
#pragma unroll
            for (int k1 = 0; k1 < NP1; k1++) row += kf_far<KT>(fmaf(gx[k1], gx[k1], dyz), q[j + k1], kp);
            j += NP1;
            kahan_add(s, c, row);
        }
    }
    return s - c;
}

template <int KT>
__device__ float pc_cluster_dispatch(int np1, float x, float y, float z, const float *g, const float *q, float kp)
{
    switch (np1) {
#define BT_CASE(N) case N: return pc_cluster<KT, N>(x, y, z, g, q, kp);
        BT_CASE(2) BT_CASE(3) BT_CASE(4) BT_CASE(5) BT_CASE(6) BT_CASE(7) BT_CASE(8)
        BT_CASE(9) BT_CASE(10) BT_CASE(11) BT_CASE(12) BT_CASE(13)
#undef BT_CASE
    }
    return 0.f;
}

// Particle-output evaluation, mixed precision.  One thread per target.
template <int KT>
__global__ void __launch_bounds__(MX_THREADS)
k_eval_targets_mixed(MixedTargetsArgs a)
{
    extern __shared__ float smf[];
    const int2 it = a.items[blockIdx.x];
    const int u = it.x;
    const int tnode = a.leaf_node[u];
    const int tb = a.t_ibeg[tnode], tn = a.t_numpar[tnode];
    const int ti = it.y * MX_THREADS + threadIdx.x;
    const bool active = ti < tn;
    const int t = tb + (active ? ti : 0);
    const float4 tp = a.tpos[t];
    const double cx = a.t_ctr[3 * tnode], cy = a.t_ctr[3 * tnode + 1], cz = a.t_ctr[3 * tnode + 2];
    const float kp = (float)a.kp;
    double acc = 0.0;

    // far field
    for (int64_t e = a.a_off[u]; e < a.a_off[u + 1]; e++) {
        const int s = a.a_idx[e];
        const int deg = a.a_deg ? a.a_deg[e] : a.n;
        const int np1 = deg + 1, P = np1 * np1 * np1;
        float *g = smf;
        float *q = smf + 3 * 16;
        const double *gs = a.s_grid[deg] + (size_t)s * 3 * np1;
        const float *Qs = a.Q32[deg] + (size_t)s * P;
        for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) {
            int ax = i / np1;
            double c = ax == 0 ? cx : ax == 1 ? cy : cz;
            g[ax * np1 + (i % np1)] = (float)(gs[i] - c);
        }
        for (int i = threadIdx.x; i < P; i += blockDim.x) q[i] = Qs[i];
        __syncthreads();
        if (active) acc += (double)pc_cluster_dispatch<KT>(np1, tp.x, tp.y, tp.z, g, q, kp);
        __syncthreads();
    }
    // near field: source leaves, particles relative to their leaf centre
    float4 *tile = reinterpret_cast<float4 *>(smf);
    for (int64_t e = a.d_off[u]; e < a.d_off[u + 1]; e++) {
        const int s = a.d_idx[e];
        const int sb = a.s_ibeg[s], sn = a.s_numpar[s];
        const float ox = (float)(a.s_ctr[3 * s] - cx), oy = (float)(a.s_ctr[3 * s + 1] - cy),
                    oz = (float)(a.s_ctr[3 * s + 2] - cz);
        const float x = tp.x - ox, y = tp.y - oy, z = tp.z - oz;   // target in the source leaf's frame
        for (int c0 = 0; c0 < sn; c0 += MX_TILE) {
            int cm = min(MX_TILE, sn - c0);
            for (int i = threadIdx.x; i < cm; i += blockDim.x) tile[i] = a.spos[sb + c0 + i];
            __syncthreads();
            if (active) {
                float s0 = 0.f, s1 = 0.f;
                int i = 0;
                for (; i + 1 < cm; i += 2) {
                    float4 p = tile[i], p1 = tile[i + 1];
                    float dx = x - p.x, dy = y - p.y, dz = z - p.z;
                    float dx1 = x - p1.x, dy1 = y - p1.y, dz1 = z - p1.z;
                    s0 += kf_pp<KT>(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), p.w, kp);
                    s1 += kf_pp<KT>(fmaf(dx1, dx1, fmaf(dy1, dy1, dz1 * dz1)), p1.w, kp);
                }
                if (i < cm) {
                    float4 p = tile[i];
                    float dx = x - p.x, dy = y - p.y, dz = z - p.z;
                    s0 += kf_pp<KT>(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), p.w, kp);
                }
                acc += (double)s0 + (double)s1;
            }
            __syncthreads();
        }
    }
    if (active) a.pot[t] = acc;
}

// Grid-output evaluation (M2L from source clusters + CP from source leaves)
// onto the grid of a target node, mixed precision, Lagrange.
template <int KT>
__global__ void __launch_bounds__(MX_THREADS)
k_eval_grids_mixed(MixedGridsArgs a)
{
    extern __shared__ float smf[];
    const int2 it = a.items[blockIdx.x];
    const int T = it.x;
    const int np1 = a.n + 1, P = np1 * np1 * np1;
    const int j0 = it.y * MX_THREADS + threadIdx.x;
    const bool active = j0 < P;
    const int jj = active ? j0 : 0;
    const double *tg = a.t_grid + (size_t)T * 3 * np1;
    const double cx = a.t_ctr[3 * T], cy = a.t_ctr[3 * T + 1], cz = a.t_ctr[3 * T + 2];
    const float x = (float)(tg[jj % np1] - cx), y = (float)(tg[np1 + (jj / np1) % np1] - cy),
                z = (float)(tg[2 * np1 + jj / (np1 * np1)] - cz);
    const float kp = (float)a.kp;
    double acc = 0.0;
    for (int64_t e = a.c_off[T]; e < a.c_off[T + 1]; e++) {
        const int s = a.c_idx[e];
        float *g = smf;
        float *q = smf + 3 * 16;
        const double *gs = a.s_grid + (size_t)s * 3 * np1;
        for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) {
            int ax = i / np1;
            double c = ax == 0 ? cx : ax == 1 ? cy : cz;
            g[ax * np1 + (i % np1)] = (float)(gs[i] - c);
        }
        for (int i = threadIdx.x; i < P; i += blockDim.x) q[i] = a.Q32[(size_t)s * P + i];
        __syncthreads();
        if (active) acc += (double)pc_cluster_dispatch<KT>(np1, x, y, z, g, q, kp);
        __syncthreads();
    }
    float4 *tile = reinterpret_cast<float4 *>(smf);
    for (int64_t e = a.p_off[T]; e < a.p_off[T + 1]; e++) {
        const int s = a.p_idx[e];
        const int sb = a.s_ibeg[s], sn = a.s_numpar[s];
        const float ox = (float)(a.s_ctr[3 * s] - cx), oy = (float)(a.s_ctr[3 * s + 1] - cy),
                    oz = (float)(a.s_ctr[3 * s + 2] - cz);
        const float xs = x - ox, ys = y - oy, zs = z - oz;
        for (int c0 = 0; c0 < sn; c0 += MX_TILE) {
            int cm = min(MX_TILE, sn - c0);
            for (int i = threadIdx.x; i < cm; i += blockDim.x) tile[i] = a.spos[sb + c0 + i];
            __syncthreads();
            if (active) {
                float s0 = 0.f;
                for (int i = 0; i < cm; i++) {
                    float4 p = tile[i];
                    float dx = xs - p.x, dy = ys - p.y, dz = zs - p.z;
                    s0 += kf_far<KT>(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), p.w, kp);
                }
                acc += (double)s0;
            }
            __syncthreads();
        }
    }
    if (active) a.Phi[(size_t)T * P + j0] = acc;
}

// Particles relative to the centre of their leaf, FP32 (x', y', z', q).
__global__ void k_rel_positions(int nleaves, const int *__restrict__ leaves, const int *__restrict__ ibeg,
                                const int *__restrict__ numpar, const double *__restrict__ ctr,
                                const double *__restrict__ x, const double *__restrict__ y,
                                const double *__restrict__ z, const double *__restrict__ q, float4 *__restrict__ out)
{
    const int l = leaves[blockIdx.x];
    const double cx = ctr[3 * l], cy = ctr[3 * l + 1], cz = ctr[3 * l + 2];
    for (int i = ibeg[l] + threadIdx.x; i < ibeg[l] + numpar[l]; i += blockDim.x)
        out[i] = make_float4((float)(x[i] - cx), (float)(y[i] - cy), (float)(z[i] - cz), q ? (float)q[i] : 0.f);
}

__global__ void k_to_f32(size_t n, const double *__restrict__ src, float *__restrict__ dst)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

void launch_rel_positions(int nleaves, const int *leaves, const int *ibeg, const int *numpar, const double *ctr,
                          const double *x, const double *y, const double *z, const double *q, float4 *out,
                          cudaStream_t st)
{
    if (nleaves > 0) k_rel_positions<<<nleaves, 256, 0, st>>>(nleaves, leaves, ibeg, numpar, ctr, x, y, z, q, out);
}

void launch_to_f32(size_t n, const double *src, float *dst, cudaStream_t st)
{
    if (n > 0) k_to_f32<<<1184, 256, 0, st>>>(n, src, dst);
}

static size_t mixed_smem(int max_np1)
{
    size_t far = sizeof(float) * (size_t)(3 * 16 + max_np1 * max_np1 * max_np1);
    size_t near = sizeof(float4) * MX_TILE;
    return far > near ? far : near;
}

template <int KT>
static void eval_targets_mixed_t(const MixedTargetsArgs &a, cudaStream_t st)
{
    size_t sm = mixed_smem(a.max_np1);
    cudaFuncSetAttribute(k_eval_targets_mixed<KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_eval_targets_mixed<KT><<<a.nitems, MX_THREADS, sm, st>>>(a);
}

void launch_eval_targets_mixed(int kernel, const MixedTargetsArgs &a, cudaStream_t st)
{
    if (a.nitems <= 0) return;
    if (kernel == 1) eval_targets_mixed_t<1>(a, st);
    else if (kernel == 2) eval_targets_mixed_t<2>(a, st);
    else eval_targets_mixed_t<3>(a, st);
}

template <int KT>
static void eval_grids_mixed_t(const MixedGridsArgs &a, cudaStream_t st)
{
    size_t sm = mixed_smem(a.n + 1);
    cudaFuncSetAttribute(k_eval_grids_mixed<KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_eval_grids_mixed<KT><<<a.nitems, MX_THREADS, sm, st>>>(a);
}

void launch_eval_grids_mixed(int kernel, const MixedGridsArgs &a, cudaStream_t st)
{
    if (a.nitems <= 0) return;
    if (kernel == 1) eval_grids_mixed_t<1>(a, st);
    else if (kernel == 2) eval_grids_mixed_t<2>(a, st);
    else eval_grids_mixed_t<3>(a, st);
}

}  // namespace bt
