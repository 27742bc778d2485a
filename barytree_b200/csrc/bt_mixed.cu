// bt_mixed.cu -- mixed-precision evaluation kernels of barytree_b200.
//
// Arithmetic: every kernel evaluation (PP, PC, CP, M2L) runs in FP32 on
// coordinates relative to the centre of the target leaf / node, so FP32 only
// ever sees displacements of the size of the interaction, never absolute
// positions.  Centre offsets between the two sides of an interaction are
// formed in FP64 and rounded once.  Per-interaction partial sums are FP32
// (far field: Kahan-compensated per grid row); they are folded into an FP64
// per-target accumulator after every list entry / tile, which is the FP64
// far+near reduction.  Tree boxes, Chebyshev node placement, exact-node
// coincidence tests and the barycentric passes stay FP64 (bt_device.cu).
//
// Throughput: the kernels are issue-bound, so each thread evaluates two
// targets against every shared-memory value it loads, the coincidence test
// of the skipping kernels runs only for source leaves whose box overlaps the
// target leaf's box, and the special functions are single MUFU instructions
// (rsqrt.approx / ex2.approx, flush-to-zero).  The far-field loops are
// instantiated per degree (NP1 = n+1) so one axis of grid coordinates lives
// in registers.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "bt_f2.cuh"
#include "bt_kernels.cuh"
#include "bt_mixed.h"

namespace bt {

// Kernel value for a well-separated pair.  kc: Yukawa -kappa*log2(e);
// regularised Coulomb eps^2; unused for Coulomb.
template <int KT>
__device__ __forceinline__ float kf_far(float r2, float q, float kc)
{
    if (KT == 1) {
        return q * rsqrt_apx(r2);
    } else if (KT == 2) {
        // one Newton step on 1/r (the MUFU estimate's error would otherwise
        // enter both 1/r and the exponent); the FMA pipe has room for it here
        float rinv = rsqrt_apx(r2);
        float h = r2 * rinv;
        float t = fmaf(-0.5f * h, rinv, 1.5f);
        float e = ex2_apx(kc * (h * t));
        return (q * (rinv * t)) * e;
    } else {
        return q * rsqrt_apx(r2 + kc);
    }
}

__device__ __forceinline__ void kahan_add(float &s, float &c, float v)
{
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

constexpr int MX_THREADS = 128;                 // threads of the grid-output kernel
// Register budget of the grid-output kernel: BT_MX_MIN_BLOCKS resident blocks
// per SM (unset: the compiler's choice).
#ifdef BT_MX_MIN_BLOCKS
#define BT_MX_BOUNDS __launch_bounds__(MX_THREADS, BT_MX_MIN_BLOCKS)
#else
#define BT_MX_BOUNDS __launch_bounds__(MX_THREADS)
#endif
constexpr int MX_TILE = 1024;                   // sources per tile of the grid-output kernel
// Register budget of the 2-targets-per-thread Lagrange particle-output
// kernel (Coulomb, regularised Coulomb): room for 6 resident blocks per SM.
// Left to itself the compiler takes 94 registers (5 blocks) for the packed
// far field, which measured 21 % slower on the 16M system; at 80 registers
// (a few bytes of spill) it runs 1.4 % faster than the scalar far field.
#ifndef BT_MX_MIN_BLOCKS_T2
#define BT_MX_MIN_BLOCKS_T2 6
#endif
// Yukawa: 6 blocks (80 registers, 24 bytes of spill) measured 2 % faster
// than the compiler's 96 registers on the 1M cluster-cluster system; for the
// Hermite kernels 5 blocks measured the same as the compiler's choice.
#ifndef BT_MX_MIN_BLOCKS_YUK
#define BT_MX_MIN_BLOCKS_YUK 6
#endif
#ifndef BT_MX_MIN_BLOCKS_HERM
#define BT_MX_MIN_BLOCKS_HERM 0
#endif
// resident-block budget of the 2-targets-per-thread kernel (0: the compiler's choice)
template <int KT, bool HERM>
__host__ __device__ constexpr int rb_blocks()
{
    return HERM ? BT_MX_MIN_BLOCKS_HERM : KT == 2 ? BT_MX_MIN_BLOCKS_YUK : BT_MX_MIN_BLOCKS_T2;
}

// Grid points of each row of the Lagrange far field (Coulomb and
// regularised Coulomb) whose 1/r comes from rsqrt_sw / f2_rsqrt_sw on the
// FP32 and integer pipes instead of the MUFU: the first BT_FAR_SW of the
// row's n+1 (k1 < BT_FAR_SW).  A far-field value needs only two FP32
// operations besides its 1/r, so the FP32 pipe has room that the MUFU
// lacks, but less than that count suggests: on the 16M clustered system
// (degrees 4 to 11, mostly 5 to 7) the evaluation took 819.8 ms with none
// on the FP32 pipe, 802.7 ms with one per row of up to 8, and 829, 863
// and 919 ms with 2, 3 and 4 of 8 (same rel-L2, 1.0e-7).  Both forms round
// alike lane by lane, so every tile shape still gives the same bits.
#ifndef BT_FAR_SW
#define BT_FAR_SW 1
#endif
__host__ __device__ constexpr bool far_sw(int k1) { return k1 < BT_FAR_SW; }

// Far field of one source cluster (degree NP1-1) for NT targets at (x,y,z),
// relative to the target centre; g = grid coordinates relative to the same
// centre, q = proxy charges (shared memory, FP32).
template <int KT, int NP1, int NT>
__device__ __forceinline__ void pc_cluster(const float *x, const float *y, const float *z, const float *g,
                                           const float *q, float kc, float *out)
{
    float gx[NT][NP1];
#pragma unroll
    for (int t = 0; t < NT; t++)
#pragma unroll
        for (int k = 0; k < NP1; k++) gx[t][k] = x[t] - g[k];
    float s[NT], c[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) { s[t] = 0.f; c[t] = 0.f; }
    int j = 0;
    for (int k3 = 0; k3 < NP1; k3++) {
        float gz = g[2 * NP1 + k3];
        for (int k2 = 0; k2 < NP1; k2++) {
            float gy = g[NP1 + k2];
            float dyz[NT], row[NT];
#pragma unroll
            for (int t = 0; t < NT; t++) {
                float dy = y[t] - gy, dz = z[t] - gz;
                dyz[t] = fmaf(dy, dy, dz * dz);
                row[t] = 0.f;
            }
#pragma unroll
            for (int k1 = 0; k1 < NP1; k1++) {
                float qq = q[j + k1];
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    const float r2 = fmaf(gx[t][k1], gx[t][k1], dyz[t]);
                    if (KT == 2) row[t] += kf_far<KT>(r2, qq, kc);
                    else if (far_sw(k1)) row[t] = fmaf(qq, rsqrt_sw(KT == 3 ? r2 + kc : r2), row[t]);
                    else row[t] = fmaf(qq, rsqrt_apx(KT == 3 ? r2 + kc : r2), row[t]);
                }
            }
            j += NP1;
#pragma unroll
            for (int t = 0; t < NT; t++) kahan_add(s[t], c[t], row[t]);
        }
    }
#pragma unroll
    for (int t = 0; t < NT; t++) out[t] = s[t] - c[t];
}

// Hermite far field of one source cluster for NT targets (FP32; moments
// q[m * P + j], m = 0..7 in the reference's order q, qx, qy, qz, qxy, qyz,
// qxz, qxyz, with qxy..qxz pre-multiplied by 3 and qxyz by 15 when staged).
// The terms of K_*_PC_Hermite (src/kernels/coulomb/coulomb_pc.c:66-138,
// yukawa/yukawa_pc.c, regularized-coulomb/regularized-coulomb_pc.c):
//   r^-1 q + r^-3 (qx dx + qy dy + qz dz) + 3 r^-5 (qxy dx dy + qyz dy dz
//   + qxz dx dz) + 15 r^-7 qxyz dx dy dz, Yukawa with exp(-kappa r) and the
//   polynomials in kappa r.  Kahan-compensated per grid row.
template <int KT, int NP1, int NT>
__device__ __forceinline__ void pc_cluster_herm(const float *x, const float *y, const float *z, const float *g,
                                                const float *q, float kc, float kp, float *out)
{
    constexpr int P = NP1 * NP1 * NP1;
    float gx[NT][NP1];
#pragma unroll
    for (int t = 0; t < NT; t++)
#pragma unroll
        for (int k = 0; k < NP1; k++) gx[t][k] = x[t] - g[k];
    float s[NT], c[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) { s[t] = 0.f; c[t] = 0.f; }
    int j = 0;
    for (int k3 = 0; k3 < NP1; k3++) {
        const float gz = g[2 * NP1 + k3];
        for (int k2 = 0; k2 < NP1; k2++) {
            const float gy = g[NP1 + k2];
            float dy[NT], dz[NT], dyz[NT], dydz[NT], row[NT];
#pragma unroll
            for (int t = 0; t < NT; t++) {
                dy[t] = y[t] - gy;
                dz[t] = z[t] - gz;
                dyz[t] = fmaf(dy[t], dy[t], dz[t] * dz[t]);
                if (KT == 3) dyz[t] += kc;
                dydz[t] = dy[t] * dz[t];
                row[t] = 0.f;
            }
#pragma unroll
            for (int k1 = 0; k1 < NP1; k1++) {
                const int jj = j + k1;
                const float q0 = q[jj], q1 = q[P + jj], q2 = q[2 * P + jj], q3 = q[3 * P + jj];
                const float q4 = q[4 * P + jj], q5 = q[5 * P + jj], q6 = q[6 * P + jj], q7 = q[7 * P + jj];
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    const float dx = gx[t][k1];
                    const float r2 = fmaf(dx, dx, dyz[t]);
                    const float rinv = rsqrt_apx(r2);
                    const float rinv2 = rinv * rinv;
                    const float dxdy = dx * dy[t], dxdz = dx * dz[t];
                    const float a1 = fmaf(q1, dx, fmaf(q2, dy[t], q3 * dz[t]));
                    const float a2 = fmaf(q4, dxdy, fmaf(q5, dydz[t], q6 * dxdz));
                    const float a3 = q7 * dxdy * dz[t];
                    if (KT == 2) {
                        // Yukawa: exp(-kappa r) (r^-1 q + r^-3 (1 + kr) a1 + r^-5 (3 + 3kr + k^2r^2) a2
                        // + r^-7 (15 + 15kr + 6k^2r^2 + k^3r^3) a3), with a2, a3 staged x3, x15
                        const float r = r2 * rinv, kr = kp * r, kr2 = kr * kr;
                        const float e = ex2_apx(kc * r);
                        const float p1 = 1.0f + kr;
                        const float p2 = fmaf(kr2, 1.0f / 3.0f, p1);                    // (3 + 3kr + k^2r^2) / 3
                        const float p3 = fmaf(kr2 * kr, 1.0f / 15.0f, fmaf(kr2, 0.4f, p1));  // (15 + 15kr + 6k^2r^2 + k^3r^3) / 15
                        const float r3 = rinv * rinv2, r5 = r3 * rinv2, r7 = r5 * rinv2;
                        row[t] = fmaf(e, fmaf(rinv, q0, fmaf(r3 * p1, a1, fmaf(r5 * p2, a2, r7 * p3 * a3))), row[t]);
                    } else {
                        const float r3 = rinv * rinv2, r5 = r3 * rinv2, r7 = r5 * rinv2;
                        row[t] = fmaf(rinv, q0, fmaf(r3, a1, fmaf(r5, a2, fmaf(r7, a3, row[t]))));
                    }
                }
            }
            j += NP1;
#pragma unroll
            for (int t = 0; t < NT; t++) kahan_add(s[t], c[t], row[t]);
        }
    }
#pragma unroll
    for (int t = 0; t < NT; t++) out[t] = s[t] - c[t];
}

// Near-field tiles.  FP32 leaf-relative coordinates carry an absolute error
// of about 6e-8 of the leaf size, a large relative error for a pair much
// closer than the leaf size, and such a pair dominates its target's
// potential.  Pairs closer than MX_CLOSE_FRAC of the two leaves' summed
// radii ("close pairs") are therefore left out of the FP32 sums and added in
// FP64 from the FP64 coordinates and charges, straight into the FP64
// per-target accumulator (an FP32 sum would also round every later term at
// the close pair's magnitude).  Close pairs occur only between leaves whose
// boxes lie within that distance (flagged per near-field entry); the other
// entries run pp_tile_far with no test at all.

// Lagrange far field with the targets in packed pairs (NT even, Coulomb and
// regularised Coulomb): pc_cluster's operations lane by lane in f32x2
// instructions (identical results); qd holds each proxy charge twice.
template <int KT, int NP1, int NT>
__device__ __forceinline__ void pc_cluster_f2(const float *x, const float *y, const float *z, const float *g,
                                              const f2_t *qd, float kc, float *out)
{
    constexpr int NPR = NT / 2;
    f2_t gx[NPR][NP1];
#pragma unroll
    for (int p = 0; p < NPR; p++)
#pragma unroll
        for (int k = 0; k < NP1; k++) gx[p][k] = f2_make(x[2 * p] - g[k], x[2 * p + 1] - g[k]);
    float s[NT], c[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) { s[t] = 0.f; c[t] = 0.f; }
    const f2_t kc2 = f2_make(kc, kc), one = f2_make(1.0f, 1.0f), zero = f2_make(0.0f, 0.0f);
    int j = 0;
    for (int k3 = 0; k3 < NP1; k3++) {
        const float gz = g[2 * NP1 + k3];
        for (int k2 = 0; k2 < NP1; k2++) {
            const float gy = g[NP1 + k2];
            f2_t dyz[NPR], row[NPR];
#pragma unroll
            for (int p = 0; p < NPR; p++) {
                const f2_t dy = f2_make(y[2 * p] - gy, y[2 * p + 1] - gy), dz = f2_make(z[2 * p] - gz, z[2 * p + 1] - gz);
                dyz[p] = f2_fma(dy, dy, f2_mul(dz, dz));
                row[p] = zero;
            }
#pragma unroll
            for (int k1 = 0; k1 < NP1; k1++) {
                const f2_t qq = qd[j + k1];
#pragma unroll
                for (int p = 0; p < NPR; p++) {
                    f2_t r2 = f2_fma(gx[p][k1], gx[p][k1], dyz[p]);
                    if (KT == 3) r2 = f2_fma(one, kc2, r2);
                    if (far_sw(k1)) {             // resolved at compile time: k1 is unrolled
                        row[p] = f2_fma(qq, f2_rsqrt_sw(r2), row[p]);
                    } else {
                        float a, b;
                        f2_split(r2, a, b);
                        row[p] = f2_fma(qq, f2_make(rsqrt_apx(a), rsqrt_apx(b)), row[p]);
                    }
                }
            }
            j += NP1;
#pragma unroll
            for (int p = 0; p < NPR; p++) {
                float lo, hi;
                f2_split(row[p], lo, hi);
                kahan_add(s[2 * p], c[2 * p], lo);
                kahan_add(s[2 * p + 1], c[2 * p + 1], hi);
            }
        }
    }
#pragma unroll
    for (int t = 0; t < NT; t++) out[t] = s[t] - c[t];
}

// Hermite far field with the targets in packed pairs (NT even, Coulomb and
// regularised Coulomb): the same operations as pc_cluster_herm lane by lane,
// in f32x2 instructions, so the results are identical and the FMA-pipe work
// per evaluation halves.  qd holds each moment twice ({q, q}, same staging
// scales as pc_cluster_herm).
template <int KT, int NP1, int NT>
__device__ __forceinline__ void pc_cluster_herm_f2(const float *x, const float *y, const float *z, const float *g,
                                                   const f2_t *qd, float kc, float *out)
{
    constexpr int P = NP1 * NP1 * NP1, NPR = NT / 2;
    f2_t gx[NPR][NP1];
#pragma unroll
    for (int p = 0; p < NPR; p++)
#pragma unroll
        for (int k = 0; k < NP1; k++) gx[p][k] = f2_make(x[2 * p] - g[k], x[2 * p + 1] - g[k]);
    float s[NT], c[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) { s[t] = 0.f; c[t] = 0.f; }
    const f2_t kc2 = f2_make(kc, kc), one = f2_make(1.0f, 1.0f), zero = f2_make(0.0f, 0.0f);
    int j = 0;
    for (int k3 = 0; k3 < NP1; k3++) {
        const float gz = g[2 * NP1 + k3];
        for (int k2 = 0; k2 < NP1; k2++) {
            const float gy = g[NP1 + k2];
            f2_t dy[NPR], dz[NPR], dyz[NPR], dydz[NPR], row[NPR];
#pragma unroll
            for (int p = 0; p < NPR; p++) {
                dy[p] = f2_make(y[2 * p] - gy, y[2 * p + 1] - gy);
                dz[p] = f2_make(z[2 * p] - gz, z[2 * p + 1] - gz);
                dyz[p] = f2_fma(dy[p], dy[p], f2_mul(dz[p], dz[p]));
                if (KT == 3) dyz[p] = f2_fma(one, kc2, dyz[p]);
                dydz[p] = f2_mul(dy[p], dz[p]);
                row[p] = zero;
            }
#pragma unroll
            for (int k1 = 0; k1 < NP1; k1++) {
                const int jj = j + k1;
                const f2_t q0 = qd[jj], q1 = qd[P + jj], q2 = qd[2 * P + jj], q3 = qd[3 * P + jj];
                const f2_t q4 = qd[4 * P + jj], q5 = qd[5 * P + jj], q6 = qd[6 * P + jj], q7 = qd[7 * P + jj];
#pragma unroll
                for (int p = 0; p < NPR; p++) {
                    const f2_t dx = gx[p][k1];
                    const f2_t r2 = f2_fma(dx, dx, dyz[p]);
                    float ra, rb;
                    f2_split(r2, ra, rb);
                    const f2_t rinv = f2_make(rsqrt_apx(ra), rsqrt_apx(rb));
                    const f2_t rinv2 = f2_mul(rinv, rinv);
                    const f2_t dxdy = f2_mul(dx, dy[p]), dxdz = f2_mul(dx, dz[p]);
                    const f2_t a1 = f2_fma(q1, dx, f2_fma(q2, dy[p], f2_mul(q3, dz[p])));
                    const f2_t a2 = f2_fma(q4, dxdy, f2_fma(q5, dydz[p], f2_mul(q6, dxdz)));
                    const f2_t a3 = f2_mul(f2_mul(q7, dxdy), dz[p]);
                    const f2_t r3 = f2_mul(rinv, rinv2), r5 = f2_mul(r3, rinv2), r7 = f2_mul(r5, rinv2);
                    row[p] = f2_fma(rinv, q0, f2_fma(r3, a1, f2_fma(r5, a2, f2_fma(r7, a3, row[p]))));
                }
            }
            j += NP1;
#pragma unroll
            for (int p = 0; p < NPR; p++) {
                float lo, hi;
                f2_split(row[p], lo, hi);
                kahan_add(s[2 * p], c[2 * p], lo);
                kahan_add(s[2 * p + 1], c[2 * p + 1], hi);
            }
        }
    }
#pragma unroll
    for (int t = 0; t < NT; t++) out[t] = s[t] - c[t];
}

// Packed far field (Lagrange and Hermite) for this kernel type and target count?
template <int KT, int NT>
__host__ __device__ constexpr bool far_packed() { return KT != 2 && NT % 2 == 0; }

// q: the staged proxy charges, as {q, q} pairs when far_packed<KT, NT>().
template <int KT, int NT>
__device__ void pc_cluster_dispatch(int np1, const float *x, const float *y, const float *z, const float *g,
                                    const float *q, float kc, float *out)
{
    switch (np1) {
#define BT_CASE(N)                                                                                         \
    case N:                                                                                                \
        if constexpr (far_packed<KT, NT>())                                                                \
            pc_cluster_f2<KT, N, NT>(x, y, z, g, reinterpret_cast<const f2_t *>(q), kc, out);              \
        else                                                                                               \
            pc_cluster<KT, N, NT>(x, y, z, g, q, kc, out);                                                 \
        return;
        BT_CASE(2) BT_CASE(3) BT_CASE(4) BT_CASE(5) BT_CASE(6) BT_CASE(7) BT_CASE(8)
        BT_CASE(9) BT_CASE(10) BT_CASE(11) BT_CASE(12) BT_CASE(13)
#undef BT_CASE
    }
#pragma unroll
    for (int t = 0; t < NT; t++) out[t] = 0.f;
}


// q: the staged moments, as {q, q} pairs when far_packed<KT, NT>().
template <int KT, int NT>
__device__ void pc_cluster_herm_dispatch(int np1, const float *x, const float *y, const float *z, const float *g,
                                         const float *q, float kc, float kp, float *out)
{
    switch (np1) {
#define BT_CASE(N)                                                                                         \
    case N:                                                                                                \
        if constexpr (far_packed<KT, NT>())                                                               \
            pc_cluster_herm_f2<KT, N, NT>(x, y, z, g, reinterpret_cast<const f2_t *>(q), kc, out);         \
        else                                                                                               \
            pc_cluster_herm<KT, N, NT>(x, y, z, g, q, kc, kp, out);                                        \
        return;
        BT_CASE(2) BT_CASE(3) BT_CASE(4) BT_CASE(5) BT_CASE(6) BT_CASE(7) BT_CASE(8)
        BT_CASE(9) BT_CASE(10) BT_CASE(11) BT_CASE(12) BT_CASE(13)
#undef BT_CASE
    }
#pragma unroll
    for (int t = 0; t < NT; t++) out[t] = 0.f;
}

// Near-field source tile in shared memory, structure of arrays (x', y', z'
// relative to the source leaf centre, q), padded to a multiple of 4 with
// charge-free sources far away.
struct Tile {
    float *x, *y, *z, *q;
};

constexpr float MX_PAD_POS = 1.0e18f;   // r2 ~ 1e36 < FLT_MAX; with q = 0 it adds nothing

// Two sources (a pair) against one target, accumulated into the pair sum S.
// kc: mixed_kernel_constant(); kc2 = {kc, kc}.
template <int KT>
__device__ __forceinline__ f2_t kf2_acc(f2_t r2, f2_t q, f2_t S, f2_t kc2)
{
    if (KT == 3) r2 = f2_fma(f2_make(1.0f, 1.0f), kc2, r2);   // r2 + eps^2
    float a, b;
    f2_split(r2, a, b);
    const f2_t rinv = f2_make(rsqrt_apx(a), rsqrt_apx(b));
    if (KT != 2) return f2_fma(q, rinv, S);
    // Yukawa as kf_far: one Newton step on 1/r, then exp(-kappa r) by ex2
    const f2_t h = f2_mul(r2, rinv);
    const f2_t t = f2_fma(f2_mul(h, f2_make(-0.5f, -0.5f)), rinv, f2_make(1.5f, 1.5f));
    float e0, e1;
    f2_split(f2_mul(kc2, f2_mul(h, t)), e0, e1);
    const f2_t e = f2_make(ex2_apx(e0), ex2_apx(e1));
    return f2_fma(q, f2_mul(f2_mul(rinv, t), e), S);
}

// One tile against the thread's TPT targets (x, y, z in the source
// leaf's frame).  NEAR: also the smallest r2 per target (mn), which tells
// whether the tile holds a close pair.
template <int KT, bool NEAR, int TPT>
__device__ __forceinline__ void pp_tile(const Tile tl, int cm4, const float *x, const float *y, const float *z,
                                        float kc, float *s, float *mn)
{
    f2_t X[TPT], Y[TPT], Z[TPT], S[TPT];
#pragma unroll
    for (int t = 0; t < TPT; t++) {
        X[t] = f2_make(x[t], x[t]);
        Y[t] = f2_make(y[t], y[t]);
        Z[t] = f2_make(z[t], z[t]);
        S[t] = f2_make(0.0f, 0.0f);
    }
    const f2_t kc2 = f2_make(kc, kc);
#pragma unroll 2
    for (int i = 0; i < cm4; i += 4) {
        const ulonglong2 PX = *reinterpret_cast<const ulonglong2 *>(tl.x + i);
        const ulonglong2 PY = *reinterpret_cast<const ulonglong2 *>(tl.y + i);
        const ulonglong2 PZ = *reinterpret_cast<const ulonglong2 *>(tl.z + i);
        const ulonglong2 PQ = *reinterpret_cast<const ulonglong2 *>(tl.q + i);
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
            const f2_t px = hh ? PX.y : PX.x, py = hh ? PY.y : PY.x, pz = hh ? PZ.y : PZ.x, pq = hh ? PQ.y : PQ.x;
#pragma unroll
            for (int t = 0; t < TPT; t++) {
                const f2_t dx = f2_sub(X[t], px), dy = f2_sub(Y[t], py), dz = f2_sub(Z[t], pz);
                const f2_t r2 = f2_fma(dx, dx, f2_fma(dy, dy, f2_mul(dz, dz)));
                if (NEAR) {
                    float a, b;
                    f2_split(r2, a, b);
                    mn[t] = fminf(mn[t], fminf(a, b));
                }
                S[t] = kf2_acc<KT>(r2, pq, S[t], kc2);
            }
        }
    }
#pragma unroll
    for (int t = 0; t < TPT; t++) {
        float a, b;
        f2_split(S[t], a, b);
        s[t] = a + b;
    }
}

// A tile holding a close pair for this target, again in scalar form: the
// FP32 sum over the pairs at or beyond the close distance (which also drops
// coincident pairs, r2 == 0), and the close pairs in FP64 from the FP64
// coordinates and charges with the reference's skipping rule (k_pp).
template <int KT>
__device__ __noinline__ float pp_tile_close(const Tile tl, int cm, float x, float y, float z, float kc, float thr2,
                                            double xd, double yd, double zd, const double *__restrict__ sx,
                                            const double *__restrict__ sy, const double *__restrict__ sz,
                                            const double *__restrict__ sq, int base, double kp, double *acc)
{
    float s = 0.0f;
    double a = 0.0;
    for (int i = 0; i < cm; i++) {
        const float dx = x - tl.x[i], dy = y - tl.y[i], dz = z - tl.z[i];
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        if (r2 >= thr2) {
            s += kf_far<KT>(r2, tl.q[i], kc);
        } else {
            const int gi = base + i;
            const double ex = xd - sx[gi], ey = yd - sy[gi], ez = zd - sz[gi];
            a += k_pp<KT>(ex * ex + ey * ey + ez * ez, sq[gi], kp);
        }
    }
    *acc += a;
    return s;
}

// Particle-output evaluation, mixed precision.  Each thread owns TPT
// targets of a work item (target leaf, chunk of MX_CHUNK targets).
// Blocks of a work-queue launch take items (cost-sorted, longest first) from
// a device counter until the queue is empty; without a queue, block b
// evaluates item b.
__device__ __forceinline__ int next_item(int *queue, int *slot)
{
    if (threadIdx.x == 0) *slot = atomicAdd(queue, 1);
    __syncthreads();
    const int w = *slot;
    __syncthreads();
    return w;
}

template <int KT, bool HERM, int TPT>
__device__ __forceinline__ void targets_item(const MixedTargetsArgs &a, const int2 it, float *smf)
{
    const int u = it.x;
    const int tnode = a.leaf_node[u];
    const int tb = a.t_ibeg[tnode], tn = a.t_numpar[tnode];
    float x[TPT], y[TPT], z[TPT];
    bool act[TPT];
    int tid[TPT];
#pragma unroll
    for (int t = 0; t < TPT; t++) {
        int ti = it.y * MX_CHUNK + t * (MX_CHUNK / TPT) + threadIdx.x;
        act[t] = ti < tn;
        tid[t] = tb + (act[t] ? ti : 0);
        float4 tp = a.tpos[tid[t]];
        x[t] = tp.x; y[t] = tp.y; z[t] = tp.z;
    }
    const double trad = a.t_rad[tnode];
    const double cx = a.t_ctr[3 * tnode], cy = a.t_ctr[3 * tnode + 1], cz = a.t_ctr[3 * tnode + 2];
    const float kc = (float)a.kc;
    double acc[TPT];
#pragma unroll
    for (int t = 0; t < TPT; t++) acc[t] = 0.0;

    // far field: source clusters
    for (int64_t e = a.a_off[u]; e < a.a_off[u + 1]; e++) {
        const int s = a.a_idx[e];
        const int deg = a.a_deg ? a.a_deg[e] : a.n;
        const int np1 = deg + 1, P = np1 * np1 * np1;
        float *g = smf;
        float *q = smf + 3 * 16;
        const double *gs = a.s_grid[deg] + (size_t)s * 3 * np1;
        for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) {
            int ax = i / np1;
            double c = ax == 0 ? cx : ax == 1 ? cy : cz;
            g[ax * np1 + (i % np1)] = (float)(gs[i] - c);
        }
        float v[TPT];
        if (HERM) {
            const float *Qs = a.Q32[deg] + (size_t)s * 8 * P;
            for (int i = threadIdx.x; i < 8 * P; i += blockDim.x) {
                const int m = i / P;
                const float v = Qs[i] * (m == 7 ? 15.0f : m >= 4 ? 3.0f : 1.0f);
                if constexpr (far_packed<KT, TPT>()) reinterpret_cast<f2_t *>(q)[i] = f2_make(v, v);
                else q[i] = v;
            }
            __syncthreads();
            pc_cluster_herm_dispatch<KT, TPT>(np1, x, y, z, g, q, kc, (float)a.kp, v);
        } else {
            const float *Qs = a.Q32[deg] + (size_t)s * P;
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                if constexpr (far_packed<KT, TPT>()) reinterpret_cast<f2_t *>(q)[i] = f2_make(Qs[i], Qs[i]);
                else q[i] = Qs[i];
            }
            __syncthreads();
            pc_cluster_dispatch<KT, TPT>(np1, x, y, z, g, q, kc, v);
        }
#pragma unroll
        for (int t = 0; t < TPT; t++) acc[t] += (double)v[t];
        __syncthreads();
    }
    // near field: source leaves, particles relative to their leaf centre
    // fixed array strides (the tile length only bounds the loop): a runtime
    // stride costs the Coulomb kernel 16 registers and a resident block
    const int tile = a.tile;
    const Tile tl{smf, smf + MX_TILE_MAX, smf + 2 * MX_TILE_MAX, smf + 3 * MX_TILE_MAX};
    for (int64_t e = a.d_off[u]; e < a.d_off[u + 1]; e++) {
        const int s = a.d_idx[e];
        const bool near = a.d_flag[e] != 0;
        const int sb = a.s_ibeg[s], sn = a.s_numpar[s];
        const float ox = (float)(a.s_ctr[3 * s] - cx), oy = (float)(a.s_ctr[3 * s + 1] - cy),
                    oz = (float)(a.s_ctr[3 * s + 2] - cz);
        float xs[TPT], ys[TPT], zs[TPT];   // targets in the source leaf's frame
#pragma unroll
        for (int t = 0; t < TPT; t++) { xs[t] = x[t] - ox; ys[t] = y[t] - oy; zs[t] = z[t] - oz; }
        // at least the smallest normal float, so that a coincident pair (r2
        // == 0 after flushing) always takes the FP64 path with the skipping
        // rule, also between single-particle leaves of radius 0
        const double rr = MX_CLOSE_FRAC * (trad + a.s_rad[s]);
        const float thr2 = fmaxf((float)(rr * rr), FLT_MIN);
        for (int c0 = 0; c0 < sn; c0 += tile) {
            const int cm = min(tile, sn - c0), cm4 = (cm + 3) & ~3;
            for (int i = threadIdx.x; i < cm4; i += blockDim.x) {
                const float4 p = i < cm ? a.spos[sb + c0 + i] : make_float4(MX_PAD_POS, MX_PAD_POS, MX_PAD_POS, 0.0f);
                tl.x[i] = p.x; tl.y[i] = p.y; tl.z[i] = p.z; tl.q[i] = p.w;
            }
            __syncthreads();
            float sum[TPT], mn[TPT];
            if (near) {
#pragma unroll
                for (int t = 0; t < TPT; t++) mn[t] = FLT_MAX;
                pp_tile<KT, true, TPT>(tl, cm4, xs, ys, zs, kc, sum, mn);
                bool close = false;
#pragma unroll
                for (int t = 0; t < TPT; t++) close |= act[t] && mn[t] < thr2;
                if (__any_sync(0xffffffffu, close)) {
#pragma unroll
                    for (int t = 0; t < TPT; t++)
                        if (act[t] && mn[t] < thr2)
                            sum[t] = pp_tile_close<KT>(tl, cm, xs[t], ys[t], zs[t], kc, thr2, a.tx64[tid[t]],
                                                       a.ty64[tid[t]], a.tz64[tid[t]], a.sx64, a.sy64, a.sz64,
                                                       a.sq64, sb + c0, a.kp, &acc[t]);
                }
            } else {
                pp_tile<KT, false, TPT>(tl, cm4, xs, ys, zs, kc, sum, mn);
            }
#pragma unroll
            for (int t = 0; t < TPT; t++) acc[t] += (double)sum[t];
            __syncthreads();
        }
    }
#pragma unroll
    for (int t = 0; t < TPT; t++)
        if (act[t]) a.pot[tid[t]] = acc[t];
}

template <int KT, bool HERM, int TPT>
__device__ __forceinline__ void eval_targets_mixed_body(const MixedTargetsArgs &a)
{
    extern __shared__ float smf[];
    __shared__ int slot;
    int w = a.queue ? next_item(a.queue, &slot) : blockIdx.x;
    while (w < a.nitems) {
        targets_item<KT, HERM, TPT>(a, a.items[w], smf);
        if (!a.queue) break;
        w = next_item(a.queue, &slot);
    }
}

template <int KT, bool HERM, int TPT>
__global__ void __launch_bounds__(MX_CHUNK / TPT) k_eval_targets_mixed(MixedTargetsArgs a)
{
    eval_targets_mixed_body<KT, HERM, TPT>(a);
}

// The same kernel under the register budget of BT_MX_MIN_BLOCKS_T2 resident
// blocks (2 targets per thread, Lagrange, Coulomb and regularised Coulomb).
template <int KT, bool HERM, int TPT>
__global__ void __launch_bounds__(MX_CHUNK / TPT, rb_blocks<KT, HERM>()) k_eval_targets_mixed_rb(MixedTargetsArgs a)
{
    eval_targets_mixed_body<KT, HERM, TPT>(a);
}

// Grid-output evaluation (M2L from source clusters + CP from source leaves)
// onto the grid of a target node, mixed precision, Lagrange.  One thread per
// target grid point.
template <int KT>
__device__ __forceinline__ void grids_item(const MixedGridsArgs &a, const int2 it, float *smf)
{
    const int T = it.x;
    const int np1 = a.n + 1, P = np1 * np1 * np1;
    const int j0 = it.y * MX_THREADS + threadIdx.x;
    const bool active = j0 < P;
    const int jj = active ? j0 : 0;
    const double *tg = a.t_grid + (size_t)T * 3 * np1;
    const double cx = a.t_ctr[3 * T], cy = a.t_ctr[3 * T + 1], cz = a.t_ctr[3 * T + 2];
    float x[1] = {(float)(tg[jj % np1] - cx)}, y[1] = {(float)(tg[np1 + (jj / np1) % np1] - cy)},
          z[1] = {(float)(tg[2 * np1 + jj / (np1 * np1)] - cz)};
    const float kc = (float)a.kc;
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
        float v[1];
        pc_cluster_dispatch<KT, 1>(np1, x, y, z, g, q, kc, v);
        acc += (double)v[0];
        __syncthreads();
    }
    float4 *tile = reinterpret_cast<float4 *>(smf);
    for (int64_t e = a.p_off[T]; e < a.p_off[T + 1]; e++) {
        const int s = a.p_idx[e];
        const int sb = a.s_ibeg[s], sn = a.s_numpar[s];
        const float ox = (float)(a.s_ctr[3 * s] - cx), oy = (float)(a.s_ctr[3 * s + 1] - cy),
                    oz = (float)(a.s_ctr[3 * s + 2] - cz);
        const float xs = x[0] - ox, ys = y[0] - oy, zs = z[0] - oz;
        for (int c0 = 0; c0 < sn; c0 += MX_TILE) {
            int cm = min(MX_TILE, sn - c0);
            for (int i = threadIdx.x; i < cm; i += blockDim.x) tile[i] = a.spos[sb + c0 + i];
            __syncthreads();
            float s0 = 0.f;
#pragma unroll 4
            for (int i = 0; i < cm; i++) {
                float4 p = tile[i];
                float dx = xs - p.x, dy = ys - p.y, dz = zs - p.z;
                s0 += kf_far<KT>(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), p.w, kc);
            }
            acc += (double)s0;
            __syncthreads();
        }
    }
    if (active) a.Phi[(size_t)T * P + j0] = acc;
}

template <int KT>
__global__ void BT_MX_BOUNDS
k_eval_grids_mixed(MixedGridsArgs a)
{
    extern __shared__ float smf[];
    __shared__ int slot;
    int w = a.queue ? next_item(a.queue, &slot) : blockIdx.x;
    while (w < a.nitems) {
        grids_item<KT>(a, a.items[w], smf);
        if (!a.queue) break;
        w = next_item(a.queue, &slot);
    }
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

int mixed_targets_chunk() { return MX_CHUNK; }

// Shared memory of the evaluation kernels: the far-field staging (grid
// coordinates and proxy charges of one cluster) or the near-field tile,
// whose four arrays sit MX_TILE_MAX floats apart in the particle-output
// kernel (tile_stride) whatever the tile length.
static size_t mixed_smem(int max_np1, bool herm, int tile_stride)
{
    // proxy charges are staged as {q, q} pairs (packed far field)
    size_t far = sizeof(float) * (size_t)(3 * 16 + (herm ? 16 : 2) * max_np1 * max_np1 * max_np1);
    size_t near = sizeof(float4) * (size_t)tile_stride;
    return far > near ? far : near;
}

// Grid of a work-queue launch: as many blocks as are resident at once.
template <typename K>
static int queue_grid(K kernel, int threads, size_t smem, int nitems)
{
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    int g = sms * (per_sm > 0 ? per_sm : 1);
    return g < nitems ? g : nitems;
}

template <int KT, bool HERM, int TPT>
static void eval_targets_mixed_t(const MixedTargetsArgs &a, cudaStream_t st)
{
    size_t sm = mixed_smem(a.max_np1, HERM, MX_TILE_MAX);
    auto kernel = k_eval_targets_mixed<KT, HERM, TPT>;
    if constexpr (TPT == 2 && rb_blocks<KT, HERM>() > 0) kernel = k_eval_targets_mixed_rb<KT, HERM, TPT>;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int grid = a.queue ? queue_grid(kernel, MX_CHUNK / TPT, sm, a.nitems) : a.nitems;
    kernel<<<grid, MX_CHUNK / TPT, sm, st>>>(a);
}

template <int KT, bool HERM>
static void eval_targets_mixed_h(const MixedTargetsArgs &a, cudaStream_t st)
{
    if (a.tpt == 1) eval_targets_mixed_t<KT, HERM, 1>(a, st);
    else if (a.tpt == 4) eval_targets_mixed_t<KT, HERM, 4>(a, st);
    else eval_targets_mixed_t<KT, HERM, 2>(a, st);
}

void launch_eval_targets_mixed(int kernel, const MixedTargetsArgs &a, cudaStream_t st)
{
    if (a.nitems <= 0) return;
    if (kernel == 1) a.herm ? eval_targets_mixed_h<1, true>(a, st) : eval_targets_mixed_h<1, false>(a, st);
    else if (kernel == 2) a.herm ? eval_targets_mixed_h<2, true>(a, st) : eval_targets_mixed_h<2, false>(a, st);
    else a.herm ? eval_targets_mixed_h<3, true>(a, st) : eval_targets_mixed_h<3, false>(a, st);
}

template <int KT>
static void eval_grids_mixed_t(const MixedGridsArgs &a, cudaStream_t st)
{
    size_t sm = mixed_smem(a.n + 1, false, MX_TILE);
    cudaFuncSetAttribute(k_eval_grids_mixed<KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int grid = a.queue ? queue_grid(k_eval_grids_mixed<KT>, MX_THREADS, sm, a.nitems) : a.nitems;
    k_eval_grids_mixed<KT><<<grid, MX_THREADS, sm, st>>>(a);
}

void launch_eval_grids_mixed(int kernel, const MixedGridsArgs &a, cudaStream_t st)
{
    if (a.nitems <= 0) return;
    if (kernel == 1) eval_grids_mixed_t<1>(a, st);
    else if (kernel == 2) eval_grids_mixed_t<2>(a, st);
    else eval_grids_mixed_t<3>(a, st);
}

double mixed_kernel_constant(int kernel, double kp)
{
    if (kernel == 2) return -kp * 1.4426950408889634;   // exp(-k r) = 2^(-k log2(e) r)
    if (kernel == 3) return kp * kp;
    return 0.0;
}

}  // namespace bt
