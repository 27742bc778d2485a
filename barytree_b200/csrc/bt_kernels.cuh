// bt_kernels.cuh -- device code of barytree_b200 (sm_100a).
//
// Kernel math follows the reference's interaction kernels:
//   PP   K_*_PP           src/kernels/coulomb/coulomb_pp.c:8-61, yukawa/yukawa_pp.c:9-57,
//                         regularized-coulomb/regularized-coulomb_pp.c:9-61
//   PC   K_*_PC_Lagrange  src/kernels/coulomb/coulomb_pc.c:9-61 (Hermite :66-138)
//   CP   K_*_CP_*         src/kernels/coulomb/coulomb_cp.c:9-184, yukawa/yukawa_cp.c:9-190
//   CC   K_*_CP_Lagrange on grid points  src/interaction_compute/interaction_compute_cc.c:121-127
// The barycentric passes (src/clusters/clusters.c:379-1514,
// src/interaction_compute/interaction_compute_downpass.c:151-1109) are written
// in separable form: every pass applies a Kronecker product of three per-axis
// (n+1)-point barycentric basis matrices, with the reference's exact-node
// coincidence rule (|d| < DBL_MIN selects that node) kept per axis.
#pragma once

#include <cfloat>
#include <cstdint>

namespace bt {

// The reference's KERNEL values (src/interface/BaryTreeInterface.h:7-22).
enum KernelType {
    K_COULOMB = 1, K_YUKAWA = 2, K_REGCOULOMB = 3, K_REGYUKAWA = 4, K_ATAN = 5,
    K_SINOVERR = 8, K_MQ = 9, K_RBSU = 10, K_RBSV = 11, K_USER = 12
};

constexpr int MAXNP = 17;   // n+1 <= 17 (degree <= 16)

struct TreeDev {
    int n;                 // nodes
    const int *ibeg, *numpar;
    const double *grid;    // per node: (n+1) x-nodes, (n+1) y-nodes, (n+1) z-nodes
};

// Particle-pair kernel with the reference's skipping rule (PP).
template <int KT>
__device__ __forceinline__ double k_pp(double r2, double q, double kp)
{
    if (KT == K_COULOMB) {
        return (r2 > DBL_MIN) ? q * rsqrt(r2) : 0.0;
    } else if (KT == K_YUKAWA) {
        double r = sqrt(r2);
        return (r > DBL_MIN) ? q * exp(-kp * r) / r : 0.0;
    } else {
        return q * rsqrt(r2 + kp * kp);
    }
}

// Kernel value without the skip test (PC, CP and M2L: well-separated pairs).
template <int KT>
__device__ __forceinline__ double k_far(double r2, double q, double kp)
{
    if (KT == K_COULOMB) {
        return q * rsqrt(r2);
    } else if (KT == K_YUKAWA) {
        double r = sqrt(r2);
        return q * exp(-kp * r) / r;
    } else {
        return q * rsqrt(r2 + kp * kp);
    }
}

// Any kernel at displacement d = target (or target grid point) - source (or
// source grid point); PP applies the reference's skipping rule.  kp, kp2 =
// kernel_params[0], [1]:
//   regularized Yukawa  q exp(-kappa r) / sqrt(r^2 + eps^2)      (kappa, eps)
//       src/kernels/regularized-yukawa/regularized-yukawa_{pp,pc,cp}.c
//   sin-over-r          q sin(k r) / r, PP skips r <= DBL_MIN     (k)
//       src/kernels/sin-over-r/sin-over-r_{pp,pc,cp}.c
//   user kernel         q exp(-k r) / r, PP skips r <= DBL_MIN    (k)
//       src/kernels/user_kernel/user_kernel_{pp,pc,cp}.c
//   RBS u / v (2-D)     +-1/(2 pi) q dy|dx / (dx^2 + dy^2 + delta^2)   (delta)
//       src/kernels/rbs-u/rbs-u_*.c, src/kernels/rbs-v/rbs-v_*.c
//   atan, MQ (1-D periodic in z, period L, width delta)           (L, delta)
//       src/kernels/atan/atan_{pp,pc}.c, src/kernels/mq/mq_{pp,pc}.c
template <int KT, bool PP>
__device__ __forceinline__ double k_any(double dx, double dy, double dz, double q, double kp, double kp2)
{
    constexpr double pi = 3.14159265358979323846;
    if (KT == K_COULOMB || KT == K_YUKAWA || KT == K_REGCOULOMB) {
        const double r2 = dx * dx + dy * dy + dz * dz;
        return PP ? k_pp<KT>(r2, q, kp) : k_far<KT>(r2, q, kp);
    } else if (KT == K_REGYUKAWA) {
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        return q * exp(-kp * r) / sqrt(r * r + kp2 * kp2);
    } else if (KT == K_SINOVERR || KT == K_USER) {
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        if (PP && !(r > DBL_MIN)) return 0.0;
        return KT == K_SINOVERR ? q * sin(kp * r) / r : q * exp(-kp * r) / r;
    } else if (KT == K_RBSU || KT == K_RBSV) {
        const double r = dx * dx + dy * dy + kp * kp;
        return KT == K_RBSU ? 1. / (2. * pi) * q * dy / r : -1. / (2. * pi) * q * dx / r;
    } else {
        double d = dz / kp;
        if (d < -0.5) d += 1.0;
        if (d > 0.5) d -= 1.0;
        if (KT == K_ATAN) {
            const double factor = sqrt(1. + 1.0 / (kp2 * kp2));
            const double wadj = 1. / (1. - kp2 / sqrt(1. + kp2 * kp2));
            return wadj * (q * (1.0 / pi * atan(factor * tan(pi * d)) - d));
        }
        const double dl2 = kp2 * kp2 / kp / kp;
        return q * (.5 * d * sqrt(1 + 4 * dl2) / sqrt(d * d + dl2) - d);
    }
}

// Hermite PC value at displacement d = target - grid point for the 8 moments
// q0..q7 = (q, qx, qy, qz, qxy, qyz, qxz, qxyz).
template <int KT>
__device__ __forceinline__ double k_pc_herm(double dx, double dy, double dz, const double *q, int P, double kp)
{
    double r2 = dx * dx + dy * dy + dz * dz;
    if (KT == K_YUKAWA) {
        double r = sqrt(r2);
        double rinv = 1.0 / r, r3inv = rinv * rinv * rinv, r5inv = r3inv * rinv * rinv, r7inv = r5inv * rinv * rinv;
        double k2 = kp * kp, k3 = kp * k2, rr2 = r * r, r3 = rr2 * r;
        return exp(-kp * r) * (rinv * q[0]
            + r3inv * (1 + kp * r) * (q[P] * dx + q[2 * P] * dy + q[3 * P] * dz)
            + r5inv * (3 + 3 * kp * r + k2 * rr2) * (q[4 * P] * dx * dy + q[5 * P] * dy * dz + q[6 * P] * dx * dz)
            + r7inv * (15 + 15 * kp * r + 6 * k2 * rr2 + k3 * r3) * q[7 * P] * dx * dy * dz);
    }
    if (KT == K_SINOVERR) {
        // src/kernels/sin-over-r/sin-over-r_pc.c:68-150
        const double r = sqrt(r2);
        if (!(r > DBL_MIN)) return 0.0;
        const double rinv = 1 / r, r2inv = rinv * rinv, r3inv = rinv * r2inv, r4inv = r2inv * r2inv,
                     r5inv = r3inv * r2inv, r6inv = r3inv * r3inv, r7inv = r4inv * r3inv;
        const double k2 = kp * kp, k3 = k2 * kp, sinr = sin(kp * r), cosr = cos(kp * r);
        return sinr * rinv * q[0]
            + (sinr * r3inv - kp * cosr * r2inv) * (q[P] * dx + q[2 * P] * dy + q[3 * P] * dz)
            + (sinr * (3 * r5inv - k2 * r3inv) - 3 * kp * cosr * r4inv)
                * (q[4 * P] * dx * dy + q[5 * P] * dy * dz + q[6 * P] * dx * dz)
            + (sinr * (15 * r7inv - 6 * k2 * r5inv) + cosr * (k3 * r4inv - 15 * kp * r6inv))
                * q[7 * P] * dx * dy * dz;
    }
    if (KT == K_REGCOULOMB) r2 += kp * kp;
    double rinv = rsqrt(r2);
    double rinv2 = rinv * rinv;
    double r3inv = rinv * rinv2, r5inv = r3inv * rinv2, r7inv = r5inv * rinv2;
    return rinv * q[0]
         + r3inv * (q[P] * dx + q[2 * P] * dy + q[3 * P] * dz)
         + 3.0 * r5inv * (q[4 * P] * dx * dy + q[5 * P] * dy * dz + q[6 * P] * dx * dz)
         + 15.0 * r7inv * q[7 * P] * dx * dy * dz;
}

// Hermite CP contribution of a source at d = source - grid point to the 8 grid moments.
template <int KT>
__device__ __forceinline__ void k_cp_herm(double dx, double dy, double dz, double q, double kp, double *o)
{
    double r2 = dx * dx + dy * dy + dz * dz;
    if (KT == K_SINOVERR) {
        // src/kernels/sin-over-r/sin-over-r_cp.c:68-175
        const double r = sqrt(r2);
        const double rinv = 1 / r, r2inv = rinv * rinv, r3inv = rinv * r2inv, r4inv = r2inv * r2inv,
                     r5inv = r3inv * r2inv, r6inv = r3inv * r3inv, r7inv = r4inv * r3inv;
        const double k2 = kp * kp, k3 = k2 * kp, sinr = sin(kp * r) * q, cosr = cos(kp * r) * q;
        const double d1 = sinr * r3inv - kp * cosr * r2inv;
        const double d2 = sinr * (3 * r5inv - k2 * r3inv) - 3 * kp * cosr * r4inv;
        const double d3 = sinr * (15 * r7inv - 6 * k2 * r5inv) + cosr * (k3 * r4inv - 15 * kp * r6inv);
        o[0] += sinr * rinv; o[1] += d1 * dx; o[2] += d1 * dy; o[3] += d1 * dz;
        o[4] += d2 * dx * dy; o[5] += d2 * dy * dz; o[6] += d2 * dx * dz; o[7] += d3 * dx * dy * dz;
        return;
    }
    if (KT == K_REGCOULOMB) r2 += kp * kp;
    if (KT == K_YUKAWA) {
        double r = sqrt(r2), r3 = r2 * r, r2inv = 1.0 / r2;
        double rinvq = q / r * exp(-kp * r);
        double r3inv = rinvq * r2inv, r5inv = r3inv * r2inv, r7inv = r5inv * r2inv;
        double k2 = kp * kp, k3 = kp * k2;
        double d1 = r3inv * (1 + kp * r);
        double d2 = r5inv * (3 + 3 * kp * r + k2 * r2);
        double d3 = r7inv * (15 + 15 * kp * r + 6 * k2 * r2 + k3 * r3);
        o[0] += rinvq; o[1] += d1 * dx; o[2] += d1 * dy; o[3] += d1 * dz;
        o[4] += d2 * dx * dy; o[5] += d2 * dy * dz; o[6] += d2 * dx * dz; o[7] += d3 * dx * dy * dz;
    } else {
        double r2inv = 1.0 / r2, rinvq = q * rsqrt(r2);
        double r3inv = rinvq * r2inv, r5inv = 3.0 * r3inv * r2inv, r7inv = r3inv * r2inv * r2inv;
        o[0] += rinvq; o[1] += r3inv * dx; o[2] += r3inv * dy; o[3] += r3inv * dz;
        o[4] += r5inv * dx * dy; o[5] += r5inv * dy * dz; o[6] += r5inv * dx * dz;
        o[7] += 15.0 * r7inv * dx * dy * dz;
    }
}

// Normalised Lagrange barycentric basis of the (n+1) nodes `nd` at point s:
// L[k] = (w_k/(s-nd_k)) / sum_j w_j/(s-nd_j), or the indicator of the node
// that s coincides with (|s-nd_k| < DBL_MIN), src/clusters/clusters.c:885-922.
__device__ __forceinline__ void lagrange_basis(int n, const double *nd, double s, double *L)
{
    double sum = 0.0;
    int ex = -1;
    for (int k = 0; k <= n; k++) {
        double d = s - nd[k];
        if (fabs(d) < DBL_MIN) ex = k;
        double w = ((k & 1) ? -1.0 : 1.0) * ((k == 0 || k == n) ? 0.5 : 1.0);
        double v = w / d;
        L[k] = v;
        sum += v;
    }
    if (ex >= 0) {
        for (int k = 0; k <= n; k++) L[k] = (k == ex) ? 1.0 : 0.0;
    } else {
        double inv = 1.0 / sum;
        for (int k = 0; k <= n; k++) L[k] *= inv;
    }
}

// Hermite barycentric pieces on one axis (src/clusters/clusters.c:1289-1344):
// A[k] = dj/d^2 + wx/d, B[k] = dj/d, both divided by sum_j A_j, with the
// exact-node rule: A = indicator, B = 0.
__device__ __forceinline__ void hermite_basis(int n, const double *nd, double s, const double *ww, double len,
                                              double *A, double *B)
{
    double sum = 0.0;
    int ex = -1;
    for (int k = 0; k <= n; k++) {
        double d = s - nd[k];
        if (fabs(d) < DBL_MIN) ex = k;
        double dj = (k == 0 || k == n) ? 0.25 : 1.0;
        double wx = -4.0 * ww[k] / len;
        double a = dj / (d * d) + wx / d;
        A[k] = a;
        B[k] = dj / d;
        sum += a;
    }
    if (ex >= 0) {
        for (int k = 0; k <= n; k++) { A[k] = (k == ex) ? 1.0 : 0.0; B[k] = 0.0; }
    } else {
        double inv = 1.0 / sum;
        for (int k = 0; k <= n; k++) { A[k] *= inv; B[k] *= inv; }
    }
}

}  // namespace bt
