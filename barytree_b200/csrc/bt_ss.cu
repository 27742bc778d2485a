// bt_ss.cu -- singularity subtraction (SS) kernels of barytree_b200, FP64.
//
// With singularity subtraction every source carries a weight w and every
// target a charge tq, and the potential at target i is
//   phi_i = sum_j (q_j - tq_i g(r)) w_j K(r)  + c * tq_i
// where g is the subtraction factor and c the correction constant:
//   Coulomb (alpha = kernel_params[0]):  K = 1/r, g = exp(-r^2/alpha^2),
//       c = 2 pi alpha^2        (src/kernels/coulomb/coulomb_ss_*.c)
//   Yukawa (kappa = kernel_params[0]):   K = exp(-kappa r)/r, g = 1,
//       c = 4 pi / kappa^2      (src/kernels/yukawa/yukawa_ss_*.c)
//   regularized Coulomb (alpha, eps = kernel_params[0..1]):
//       K = 1/sqrt(r^2+eps^2), g = exp(-r^2/alpha^2), c = 2 pi alpha^2
//       (src/kernels/regularized-coulomb/regularized-coulomb_ss_*.c)
//   regularized Yukawa (kappa, eps): K = exp(-kappa r)/sqrt(r^2+eps^2),
//       g = 1, c = 4 pi / kappa^2, particle-cluster Lagrange only
//       (src/kernels/regularized-yukawa/regularized-yukawa_ss_*.c)
// Source clusters carry two proxy arrays: Q from q*w and W from w (the same
// upward pass applied to both, src/clusters/clusters.c:162-200).  PC uses
// (Q_k - tq W_k g) K; target grids carry two fields, Phi_q from q*w (or Q)
// and Phi_w from g*w (or g*W), which the downward pass combines per target
// as Phi_q - tq Phi_w (interaction_compute_downpass.c:683-800).  Near-field
// pairs with r <= DBL_MIN are skipped for Coulomb and Yukawa; the
// regularized kernel never skips.  CP and CC with SS exist for Coulomb and
// Yukawa with Lagrange only, as in the reference.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdint>

#include "bt_kernels.cuh"
#include "bt_ss.h"

namespace bt {

namespace {

constexpr int SS_THREADS = 128;
constexpr int SS_TILE = 256;

// SS near-field pair (PP): target charge tq, source (q, w).
template <int KT>
__device__ __forceinline__ double ss_pp(double dx, double dy, double dz, double q, double w, double tq,
                                        double kp, double kp2)
{
    if (KT == K_COULOMB) {
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        return r > DBL_MIN ? (q - tq * exp(-r * r / (kp * kp))) * w / r : 0.0;
    } else if (KT == K_YUKAWA) {
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        return r > DBL_MIN ? (q - tq) * w * exp(-kp * r) / r : 0.0;
    } else if (KT == K_REGYUKAWA) {
        // regularized-yukawa_ss_pp.c: never skips
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        return (q - tq) * w * exp(-kp * r) / sqrt(r * r + kp2 * kp2);
    } else {
        const double r2 = dx * dx + dy * dy + dz * dz;
        return (q - tq * exp(-r2 / (kp * kp))) * w / sqrt(r2 + kp2 * kp2);
    }
}

// SS particle-cluster term of one Lagrange grid point (Q, W at the point).
template <int KT>
__device__ __forceinline__ double ss_pc(double dx, double dy, double dz, double Qk, double Wk, double tq,
                                        double kp, double kp2)
{
    if (KT == K_COULOMB) {
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        return (Qk - tq * Wk * exp(-r * r / (kp * kp))) / r;
    } else if (KT == K_YUKAWA) {
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        return (Qk - tq * Wk) * exp(-kp * r) / r;
    } else if (KT == K_REGYUKAWA) {
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        return (Qk - tq * Wk) * exp(-kp * r) / sqrt(r * r + kp2 * kp2);
    } else {
        const double r2 = dx * dx + dy * dy + dz * dz;
        return (Qk - tq * Wk * exp(-r2 / (kp * kp))) / sqrt(r2 + kp2 * kp2);
    }
}

// SS Hermite particle-cluster term: Q part as the skipping kernel, W part
// weighted by the subtraction factor (coulomb_ss_pc.c:66-166,
// yukawa_ss_pc.c:70-170, regularized-coulomb_ss_pc.c:66-166).  Q, W point
// at moment 0 of the grid point, moments P apart.
template <int KT>
__device__ __forceinline__ double ss_pc_herm(double dx, double dy, double dz, const double *Q, const double *W,
                                             int P, double tq, double kp, double kp2)
{
    if (KT == K_YUKAWA) {
        double d[8];
        for (int m = 0; m < 8; m++) d[m] = Q[m * P] - W[m * P] * tq;
        return k_pc_herm<K_YUKAWA>(dx, dy, dz, d, 1, kp);
    }
    const double eps2 = KT == K_REGCOULOMB ? kp2 * kp2 : 0.0;
    const double q_part = KT == K_REGCOULOMB ? k_pc_herm<K_REGCOULOMB>(dx, dy, dz, Q, P, kp2)
                                             : k_pc_herm<K_COULOMB>(dx, dy, dz, Q, P, kp);
    const double r = sqrt(dx * dx + dy * dy + dz * dz + eps2);
    const double r2 = r * r, rinv = 1.0 / r, r3inv = rinv * rinv * rinv, r5inv = r3inv * rinv * rinv,
                 r7inv = r5inv * rinv * rinv;
    const double a2 = r2 / (kp * kp), a4 = a2 * a2, a6 = a4 * a2;
    const double w_part = exp(-a2) * (rinv * W[0]
        + r3inv * (1 + 2 * a2) * (W[P] * dx + W[2 * P] * dy + W[3 * P] * dz)
        + r5inv * (3 + 4 * a2 + 4 * a4) * (W[4 * P] * dx * dy + W[5 * P] * dy * dz + W[6 * P] * dx * dz)
        + r7inv * (15 + 18 * a2 + 12 * a4 + 8 * a6) * W[7 * P] * dx * dy * dz);
    return q_part - tq * w_part;
}

// Contributions of a source (or a source-cluster grid point) to the two SS
// grid fields: field_q += qw K(r), field_w += w g(r) K(r).
template <int KT>
__device__ __forceinline__ void ss_grid(double dx, double dy, double dz, double qw, double w, double kp, double &fq,
                                        double &fw)
{
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (KT == K_COULOMB) {
        fq += qw / r;
        fw += exp(-r * r / (kp * kp)) * w / r;
    } else {
        const double e = exp(-kp * r) / r;
        fq += qw * e;
        fw += w * e;
    }
}

// Particle-output evaluation with SS: PC + PP per target leaf chunk, one
// target per thread (FP64).
template <int KT, bool HERM>
__global__ void __launch_bounds__(SS_THREADS) k_ss_targets(SsTargetsArgs a)
{
    __shared__ double g[3 * MAXNP];
    __shared__ double tile[5][SS_TILE];
    const int2 it = a.items[blockIdx.x];
    const int u = it.x;
    const int tnode = a.leaf_node[u];
    const int tb = a.t_ibeg[tnode], tn = a.t_numpar[tnode];
    const int ti = it.y * SS_THREADS + threadIdx.x;
    const bool active = ti < tn;
    const int t = tb + (active ? ti : 0);
    const double x = a.tx[t], y = a.ty[t], z = a.tz[t], tq = a.tq[t];
    const int np1 = a.n + 1, P = np1 * np1 * np1, nq = HERM ? 8 * P : P;
    double acc = 0.0;
    for (int64_t e = a.a_off[u]; e < a.a_off[u + 1]; e++) {
        const int s = a.a_idx[e];
        for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) g[i] = a.s_grid[(size_t)s * 3 * np1 + i];
        __syncthreads();
        if (active) {
            const double *Qs = a.Q + (size_t)s * nq, *Ws = a.W + (size_t)s * nq;
            int j = 0;
            for (int k3 = 0; k3 < np1; k3++) {
                const double dz = z - g[2 * np1 + k3];
                for (int k2 = 0; k2 < np1; k2++) {
                    const double dy = y - g[np1 + k2];
                    for (int k1 = 0; k1 < np1; k1++, j++) {
                        const double dx = x - g[k1];
                        if (HERM) acc += ss_pc_herm<KT>(dx, dy, dz, Qs + j, Ws + j, P, tq, a.kp, a.kp2);
                        else acc += ss_pc<KT>(dx, dy, dz, Qs[j], Ws[j], tq, a.kp, a.kp2);
                    }
                }
            }
        }
        __syncthreads();
    }
    for (int64_t e = a.d_off[u]; e < a.d_off[u + 1]; e++) {
        const int s = a.d_idx[e];
        const int sb = a.s_ibeg[s], sn = a.s_numpar[s];
        for (int c0 = 0; c0 < sn; c0 += SS_TILE) {
            const int cm = min(SS_TILE, sn - c0);
            for (int i = threadIdx.x; i < cm; i += blockDim.x) {
                const int k = sb + c0 + i;
                tile[0][i] = a.sx[k]; tile[1][i] = a.sy[k]; tile[2][i] = a.sz[k];
                tile[3][i] = a.sq[k]; tile[4][i] = a.sw[k];
            }
            __syncthreads();
            if (active)
                for (int i = 0; i < cm; i++)
                    acc += ss_pp<KT>(x - tile[0][i], y - tile[1][i], z - tile[2][i], tile[3][i], tile[4][i], tq, a.kp,
                                     a.kp2);
            __syncthreads();
        }
    }
    if (active) a.pot[t] = acc;
}

// Grid-output evaluation with SS (Lagrange): M2L from source clusters (Q, W)
// and CP from source particles (q*w, w) onto both fields of a target node's
// grid, one grid point per thread.
template <int KT>
__global__ void __launch_bounds__(SS_THREADS) k_ss_grids(SsGridsArgs a)
{
    __shared__ double g[3 * MAXNP];
    __shared__ double tile[5][SS_TILE];
    const int2 it = a.items[blockIdx.x];
    const int T = it.x;
    const int np1 = a.n + 1, P = np1 * np1 * np1;
    const int j0 = it.y * SS_THREADS + threadIdx.x;
    const bool active = j0 < P;
    const int jj = active ? j0 : 0;
    const double *tg = a.t_grid + (size_t)T * 3 * np1;
    const double x = tg[jj % np1], y = tg[np1 + (jj / np1) % np1], z = tg[2 * np1 + jj / (np1 * np1)];
    double fq = 0.0, fw = 0.0;
    for (int64_t e = a.c_off[T]; e < a.c_off[T + 1]; e++) {
        const int s = a.c_idx[e];
        for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) g[i] = a.s_grid[(size_t)s * 3 * np1 + i];
        __syncthreads();
        if (active) {
            const double *Qs = a.Q + (size_t)s * P, *Ws = a.W + (size_t)s * P;
            int j = 0;
            for (int k3 = 0; k3 < np1; k3++)
                for (int k2 = 0; k2 < np1; k2++)
                    for (int k1 = 0; k1 < np1; k1++, j++)
                        ss_grid<KT>(x - g[k1], y - g[np1 + k2], z - g[2 * np1 + k3], Qs[j], Ws[j], a.kp, fq, fw);
        }
        __syncthreads();
    }
    for (int64_t e = a.p_off[T]; e < a.p_off[T + 1]; e++) {
        const int s = a.p_idx[e];
        const int sb = a.s_ibeg[s], sn = a.s_numpar[s];
        for (int c0 = 0; c0 < sn; c0 += SS_TILE) {
            const int cm = min(SS_TILE, sn - c0);
            for (int i = threadIdx.x; i < cm; i += blockDim.x) {
                const int k = sb + c0 + i;
                tile[0][i] = a.sx[k]; tile[1][i] = a.sy[k]; tile[2][i] = a.sz[k];
                tile[3][i] = a.sq[k] * a.sw[k]; tile[4][i] = a.sw[k];
            }
            __syncthreads();
            if (active)
                for (int i = 0; i < cm; i++)
                    ss_grid<KT>(x - tile[0][i], y - tile[1][i], z - tile[2][i], tile[3][i], tile[4][i], a.kp, fq, fw);
            __syncthreads();
        }
    }
    if (active) {
        a.Phi_q[(size_t)T * P + j0] = fq;
        a.Phi_w[(size_t)T * P + j0] = fw;
    }
}

__global__ void k_mul(int n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) c[i] = a[i] * b[i];
}

__global__ void k_axpy(int n, double c, const double *__restrict__ x, double *__restrict__ y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += c * x[i];
}

// The correction over work items (unit, chunk of `chunk` targets): a
// target-sharded call adds it to the targets of its own leaves only.  The
// same operation as k_axpy, target by target.
__global__ void k_axpy_items(const int2 *__restrict__ items, int chunk, const int *__restrict__ leaf_node,
                             const int *__restrict__ ibeg, const int *__restrict__ numpar, double c,
                             const double *__restrict__ x, double *__restrict__ y)
{
    const int2 it = items[blockIdx.x];
    const int node = leaf_node[it.x];
    const int end = min(numpar[node], (it.y + 1) * chunk);
    for (int i = it.y * chunk + threadIdx.x; i < end; i += blockDim.x) {
        const int t = ibeg[node] + i;
        y[t] += c * x[t];
    }
}

// SS direct sum over all sources (InteractionCompute_Direct with
// singularity subtraction, src/interaction_compute/interaction_compute_direct.c:26-231):
// one target per thread, sources staged through shared memory.
template <int KT>
__global__ void __launch_bounds__(SS_THREADS)
k_ss_direct(int nt, int ns, const double *__restrict__ tx, const double *__restrict__ ty,
            const double *__restrict__ tz, const double *__restrict__ tq, const double *__restrict__ sx,
            const double *__restrict__ sy, const double *__restrict__ sz, const double *__restrict__ sq,
            const double *__restrict__ sw, double kp, double kp2, double *__restrict__ out)
{
    __shared__ double s_x[SS_TILE], s_y[SS_TILE], s_z[SS_TILE], s_q[SS_TILE], s_w[SS_TILE];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = t < nt;
    const double x = active ? tx[t] : 0.0, y = active ? ty[t] : 0.0, z = active ? tz[t] : 0.0;
    const double q = active ? tq[t] : 0.0;
    double acc = 0.0;
    for (int c0 = 0; c0 < ns; c0 += SS_TILE) {
        const int cm = min(SS_TILE, ns - c0);
        for (int i = threadIdx.x; i < cm; i += blockDim.x) {
            s_x[i] = sx[c0 + i]; s_y[i] = sy[c0 + i]; s_z[i] = sz[c0 + i];
            s_q[i] = sq[c0 + i]; s_w[i] = sw[c0 + i];
        }
        __syncthreads();
        for (int i = 0; i < cm; i++)
            acc += ss_pp<KT>(x - s_x[i], y - s_y[i], z - s_z[i], s_q[i], s_w[i], q, kp, kp2);
        __syncthreads();
    }
    if (active) out[t] = acc;
}

template <int KT, bool HERM>
void ss_targets_t(const SsTargetsArgs &a, cudaStream_t st)
{
    k_ss_targets<KT, HERM><<<a.nitems, SS_THREADS, 0, st>>>(a);
}

}  // namespace

int ss_chunk() { return SS_THREADS; }

void launch_ss_targets(int kernel, bool hermite, const SsTargetsArgs &a, cudaStream_t st)
{
    if (a.nitems <= 0) return;
    if (kernel == K_COULOMB) hermite ? ss_targets_t<K_COULOMB, true>(a, st) : ss_targets_t<K_COULOMB, false>(a, st);
    else if (kernel == K_YUKAWA) hermite ? ss_targets_t<K_YUKAWA, true>(a, st) : ss_targets_t<K_YUKAWA, false>(a, st);
    else if (kernel == K_REGYUKAWA) ss_targets_t<K_REGYUKAWA, false>(a, st);
    else hermite ? ss_targets_t<K_REGCOULOMB, true>(a, st) : ss_targets_t<K_REGCOULOMB, false>(a, st);
}

void launch_ss_grids(int kernel, const SsGridsArgs &a, cudaStream_t st)
{
    if (a.nitems <= 0) return;
    if (kernel == K_COULOMB) k_ss_grids<K_COULOMB><<<a.nitems, SS_THREADS, 0, st>>>(a);
    else k_ss_grids<K_YUKAWA><<<a.nitems, SS_THREADS, 0, st>>>(a);
}

bool ss_direct_kernel(int kernel)
{
    return kernel == K_COULOMB || kernel == K_YUKAWA || kernel == K_REGCOULOMB || kernel == K_REGYUKAWA;
}

void launch_ss_direct(int kernel, int nt, int ns, const double *tx, const double *ty, const double *tz,
                      const double *tq, const double *sx, const double *sy, const double *sz, const double *sq,
                      const double *sw, double kp, double kp2, double *out, cudaStream_t st)
{
    if (nt <= 0) return;
    const int grid = (nt + SS_THREADS - 1) / SS_THREADS;
#define BT_SSD(K) k_ss_direct<K><<<grid, SS_THREADS, 0, st>>>(nt, ns, tx, ty, tz, tq, sx, sy, sz, sq, sw, kp, kp2, out)
    if (kernel == K_COULOMB) BT_SSD(K_COULOMB);
    else if (kernel == K_YUKAWA) BT_SSD(K_YUKAWA);
    else if (kernel == K_REGYUKAWA) BT_SSD(K_REGYUKAWA);
    else BT_SSD(K_REGCOULOMB);
#undef BT_SSD
}

void launch_mul(int n, const double *a, const double *b, double *c, cudaStream_t st)
{
    if (n > 0) k_mul<<<(n + 255) / 256, 256, 0, st>>>(n, a, b, c);
}

void launch_ss_correction(int n, double c, const double *tq, double *pot, cudaStream_t st)
{
    if (n > 0) k_axpy<<<(n + 255) / 256, 256, 0, st>>>(n, c, tq, pot);
}

void launch_ss_correction_items(int nitems, const int2 *items, int chunk, const int *leaf_node, const int *ibeg,
                                const int *numpar, double c, const double *tq, double *pot, cudaStream_t st)
{
    if (nitems > 0) k_axpy_items<<<nitems, SS_THREADS, 0, st>>>(items, chunk, leaf_node, ibeg, numpar, c, tq, pot);
}

double ss_correction_constant(int kernel, double kp)
{
    const double pi = 3.14159265358979323846;
    if (kernel == K_YUKAWA || kernel == K_REGYUKAWA) return 4.0 * pi / kp / kp;
    return 2.0 * pi * kp * kp;
}

}  // namespace bt
