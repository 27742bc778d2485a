// bt_device.cu -- FP64 CUDA kernels of barytree_b200: upward pass, particle-
// and grid-output evaluations, downward pass, and the direct sum.
//
// Layouts in HBM (all FP64, structure of arrays):
//   particles: x, y, z, q in tree order (sources) / batch order (targets)
//   grids:     per node 3*(n+1) Chebyshev coordinates (x nodes, y nodes, z nodes)
//   charges:   Lagrange Q[node*P + j], Hermite Q[(node*8 + m)*P + j], with
//              j = k1 + (n+1)*(k2 + (n+1)*k3) (x fastest, src/clusters/clusters.c:929-933)
//   potentials on target grids: same layout as charges.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include <cfloat>
#include <cstdint>

#include "bt_device.h"
#include "bt_kernels.cuh"

namespace bt {

// ---------------------------------------------------------------------------
// Upward pass
// ---------------------------------------------------------------------------

// P2M at source leaves, Lagrange (pc_comp_ms_modifiedF, src/clusters/clusters.c:800-1004):
//   Q[k1,k2,k3] = sum_i Lx_i[k1] Ly_i[k2] Lz_i[k3] q_i.
// One CTA per leaf; each thread owns up to MAXJ grid points; particles are
// processed in chunks whose normalised bases are staged in shared memory.
constexpr int P2M_THREADS = 256;
constexpr int P2M_MAXJ = 9;      // P <= 2304  (degree <= 12)
constexpr int P2M_CHUNK = 32;

__global__ void __launch_bounds__(P2M_THREADS)
k_p2m_lagrange(int n, const int *__restrict__ leaves, const int *__restrict__ ibeg, const int *__restrict__ numpar,
               const double *__restrict__ grid, const double *__restrict__ sx, const double *__restrict__ sy,
               const double *__restrict__ sz, const double *__restrict__ sq, double *__restrict__ Q)
{
    const int node = leaves[blockIdx.x];
    const int np1 = n + 1, P = np1 * np1 * np1;
    __shared__ double nodes[3 * MAXNP];
    __shared__ double Lb[P2M_CHUNK][3][MAXNP];
    __shared__ double qs[P2M_CHUNK];
    for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) nodes[i] = grid[(size_t)node * 3 * np1 + i];
    double acc[P2M_MAXJ];
    int k1v[P2M_MAXJ], k2v[P2M_MAXJ], k3v[P2M_MAXJ];
#pragma unroll
    for (int jj = 0; jj < P2M_MAXJ; jj++) {
        acc[jj] = 0.0;
        int j = threadIdx.x + jj * P2M_THREADS;
        k1v[jj] = j % np1; k2v[jj] = (j / np1) % np1; k3v[jj] = j / (np1 * np1);
    }
    __syncthreads();
    const int b = ibeg[node], m = numpar[node];
    for (int c0 = 0; c0 < m; c0 += P2M_CHUNK) {
        int cm = min(P2M_CHUNK, m - c0);
        for (int w = threadIdx.x; w < cm * 3; w += blockDim.x) {
            int i = w / 3, a = w % 3;
            const double *src = a == 0 ? sx : a == 1 ? sy : sz;
            double s = src[b + c0 + i];
            double L[MAXNP];
            lagrange_basis(n, nodes + a * np1, s, L);
            for (int k = 0; k <= n; k++) Lb[i][a][k] = L[k];
            if (a == 0) qs[i] = sq[b + c0 + i];
        }
        __syncthreads();
#pragma unroll
        for (int jj = 0; jj < P2M_MAXJ; jj++) {
            int j = threadIdx.x + jj * P2M_THREADS;
            if (j < P) {
                double a = acc[jj];
                for (int i = 0; i < cm; i++)
                    a += Lb[i][0][k1v[jj]] * (Lb[i][1][k2v[jj]] * (Lb[i][2][k3v[jj]] * qs[i]));
                acc[jj] = a;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int jj = 0; jj < P2M_MAXJ; jj++) {
        int j = threadIdx.x + jj * P2M_THREADS;
        if (j < P) Q[(size_t)node * P + j] = acc[jj];
    }
}

// P2M in separable form.  Q[k1,k2,k3] = sum_i (q_i Lx_i[k1]) (Ly_i[k2] Lz_i[k3]):
// each thread owns whole (k2,k3) columns with all n+1 k1 entries in
// registers, so per particle it forms one product Ly*Lz and n+1 FMAs against
// q*Lx values that every thread of the warp reads from the same shared
// address.  FP64, with the exact-node rule inside lagrange_basis.
constexpr int P2S_THREADS = 128;
constexpr int P2S_CHUNK = 64;

template <int NP1>
__global__ void __launch_bounds__(P2S_THREADS)
k_p2m_sep(const int *__restrict__ leaves, const int *__restrict__ ibeg, const int *__restrict__ numpar,
          const double *__restrict__ grid, const double *__restrict__ sx, const double *__restrict__ sy,
          const double *__restrict__ sz, const double *__restrict__ sq, double *__restrict__ Q)
{
    constexpr int n = NP1 - 1, COLS = NP1 * NP1, P = COLS * NP1;
    constexpr int CPT = (COLS + P2S_THREADS - 1) / P2S_THREADS;
    const int node = leaves[blockIdx.x];
    __shared__ double nodes[3 * NP1];
    __shared__ double A[P2S_CHUNK][NP1], Ly[P2S_CHUNK][NP1], Lz[P2S_CHUNK][NP1];
    for (int i = threadIdx.x; i < 3 * NP1; i += blockDim.x) nodes[i] = grid[(size_t)node * 3 * NP1 + i];
    double acc[CPT][NP1];
    int k2[CPT], k3[CPT];
#pragma unroll
    for (int c = 0; c < CPT; c++) {
        const int col = threadIdx.x + c * P2S_THREADS;
        k2[c] = col < COLS ? col % NP1 : 0;
        k3[c] = col < COLS ? col / NP1 : 0;
#pragma unroll
        for (int k = 0; k < NP1; k++) acc[c][k] = 0.0;
    }
    __syncthreads();
    const int b = ibeg[node], m = numpar[node];
    for (int c0 = 0; c0 < m; c0 += P2S_CHUNK) {
        const int cm = min(P2S_CHUNK, m - c0);
        for (int w = threadIdx.x; w < cm * 3; w += blockDim.x) {
            const int i = w / 3, ax = w % 3;
            const double *src = ax == 0 ? sx : ax == 1 ? sy : sz;
            double L[MAXNP];
            lagrange_basis(n, nodes + ax * NP1, src[b + c0 + i], L);
            if (ax == 0) {
                const double qi = sq[b + c0 + i];
#pragma unroll
                for (int k = 0; k < NP1; k++) A[i][k] = qi * L[k];
            } else {
                double *dst = ax == 1 ? Ly[i] : Lz[i];
#pragma unroll
                for (int k = 0; k < NP1; k++) dst[k] = L[k];
            }
        }
        __syncthreads();
        for (int i = 0; i < cm; i++) {
#pragma unroll
            for (int c = 0; c < CPT; c++) {
                const double bb = Ly[i][k2[c]] * Lz[i][k3[c]];
#pragma unroll
                for (int k = 0; k < NP1; k++) acc[c][k] = fma(A[i][k], bb, acc[c][k]);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int c = 0; c < CPT; c++) {
        const int col = threadIdx.x + c * P2S_THREADS;
        if (col < COLS) {
#pragma unroll
            for (int k = 0; k < NP1; k++) Q[(size_t)node * P + k + NP1 * col] = acc[c][k];
        }
    }
}

// Per-axis basis matrix M[i][k] = L_k(child node i) of a parent grid
// evaluated at a child's grid coordinates, for all three axes, into smem.
__device__ void axis_matrices(int n, const double *pnodes, const double *cnodes, double *M)
{
    const int np1 = n + 1;
    for (int w = threadIdx.x; w < 3 * np1; w += blockDim.x) {
        int a = w / np1, i = w % np1;
        double L[MAXNP];
        lagrange_basis(n, pnodes + a * np1, cnodes[a * np1 + i], L);
        for (int k = 0; k <= n; k++) M[(a * np1 + i) * np1 + k] = L[k];
    }
}

// Separable apply: out[k] (+)= sum_i Mx[i1][k1] My[i2][k2] Mz[i3][k3] in[i]  (transpose=true, M2M)
//                  out[i] (+)= sum_k Mx[i1][k1] My[i2][k2] Mz[i3][k3] in[k]  (transpose=false, L2L)
// in, out, t1, t2 in shared memory; M = three (n+1)x(n+1) matrices [axis][i][k].
__device__ void kron_apply(int n, const double *M, const double *in, double *t1, double *t2, double *out,
                           bool transpose)
{
    const int np1 = n + 1, P = np1 * np1 * np1;
    // axis x
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
        int a1 = j % np1, rest = j / np1;
        double s = 0.0;
        for (int b1 = 0; b1 < np1; b1++) {
            double m = transpose ? M[(0 * np1 + b1) * np1 + a1] : M[(0 * np1 + a1) * np1 + b1];
            s += m * in[b1 + np1 * rest];
        }
        t1[j] = s;
    }
    __syncthreads();
    // axis y
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
        int a1 = j % np1, a2 = (j / np1) % np1, a3 = j / (np1 * np1);
        double s = 0.0;
        for (int b2 = 0; b2 < np1; b2++) {
            double m = transpose ? M[(1 * np1 + b2) * np1 + a2] : M[(1 * np1 + a2) * np1 + b2];
            s += m * t1[a1 + np1 * (b2 + np1 * a3)];
        }
        t2[j] = s;
    }
    __syncthreads();
    // axis z
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
        int a12 = j % (np1 * np1), a3 = j / (np1 * np1);
        double s = 0.0;
        for (int b3 = 0; b3 < np1; b3++) {
            double m = transpose ? M[(2 * np1 + b3) * np1 + a3] : M[(2 * np1 + a3) * np1 + b3];
            s += m * t2[a12 + np1 * np1 * b3];
        }
        out[j] += s;
    }
    __syncthreads();
}

// M2M for the parents of one level (pc_comp_ms_modifiedF_child_to_parent,
// src/clusters/clusters.c:379-582): Q[parent] = sum_children kron(M^T) Q[child].
__global__ void k_m2m(int n, const int *__restrict__ parents, const int *__restrict__ nchild,
                      const int *__restrict__ child, const double *__restrict__ grid, double *__restrict__ Q)
{
    extern __shared__ double sm[];
    const int np1 = n + 1, P = np1 * np1 * np1;
    const int p = parents[blockIdx.x];
    double *M = sm;                        // 3*np1*np1
    double *in = M + 3 * np1 * np1;        // P
    double *t1 = in + P, *t2 = t1 + P, *acc = t2 + P;
    for (int j = threadIdx.x; j < P; j += blockDim.x) acc[j] = 0.0;
    const double *pn = grid + (size_t)p * 3 * np1;
    for (int c = 0; c < nchild[p]; c++) {
        int ch = child[8 * p + c];
        axis_matrices(n, pn, grid + (size_t)ch * 3 * np1, M);
        for (int j = threadIdx.x; j < P; j += blockDim.x) in[j] = Q[(size_t)ch * P + j];
        __syncthreads();
        kron_apply(n, M, in, t1, t2, acc, true);
    }
    for (int j = threadIdx.x; j < P; j += blockDim.x) Q[(size_t)p * P + j] = acc[j];
}

// L2L for the parents of one level (cp_comp_pot_parent_to_child,
// src/interaction_compute/interaction_compute_downpass.c:151-323):
// Phi[child] += kron(M) Phi[parent].
__global__ void k_l2l(int n, const int *__restrict__ parents, const int *__restrict__ nchild,
                      const int *__restrict__ child, const double *__restrict__ grid, double *__restrict__ Phi)
{
    extern __shared__ double sm[];
    const int np1 = n + 1, P = np1 * np1 * np1;
    const int p = parents[blockIdx.x];
    double *M = sm;
    double *in = M + 3 * np1 * np1;
    double *t1 = in + P, *t2 = t1 + P, *acc = t2 + P;
    for (int j = threadIdx.x; j < P; j += blockDim.x) in[j] = Phi[(size_t)p * P + j];
    const double *pn = grid + (size_t)p * 3 * np1;
    for (int c = 0; c < nchild[p]; c++) {
        int ch = child[8 * p + c];
        axis_matrices(n, pn, grid + (size_t)ch * 3 * np1, M);
        for (int j = threadIdx.x; j < P; j += blockDim.x) acc[j] = Phi[(size_t)ch * P + j];
        __syncthreads();
        kron_apply(n, M, in, t1, t2, acc, false);
        for (int j = threadIdx.x; j < P; j += blockDim.x) Phi[(size_t)ch * P + j] = acc[j];
        __syncthreads();
    }
}

// Hermite P2M at every source node (pc_comp_ms_modifiedF_hermite,
// src/clusters/clusters.c:1224-1514): 8 moments
//   m = (AAA, BAA, ABA, AAB, BBA, ABB, BAB, BBB) x q.
constexpr int HP2M_THREADS = 512;
constexpr int HP2M_MAXJ = 5;     // P <= 2560 (degree <= 12)
constexpr int HP2M_CHUNK = 16;

__global__ void __launch_bounds__(HP2M_THREADS)
k_p2m_hermite(int n, const int *__restrict__ ibeg, const int *__restrict__ numpar, const double *__restrict__ grid,
              const double *__restrict__ box_len, const double *__restrict__ ww,
              const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ sz,
              const double *__restrict__ sq, double *__restrict__ Q)
{
    const int node = blockIdx.x;
    const int np1 = n + 1, P = np1 * np1 * np1;
    __shared__ double nodes[3 * MAXNP], wws[MAXNP], len[3];
    __shared__ double Ab[HP2M_CHUNK][3][MAXNP], Bb[HP2M_CHUNK][3][MAXNP];
    __shared__ double qs[HP2M_CHUNK];
    for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) nodes[i] = grid[(size_t)node * 3 * np1 + i];
    for (int i = threadIdx.x; i < np1; i += blockDim.x) wws[i] = ww[i];
    if (threadIdx.x < 3) len[threadIdx.x] = box_len[node * 3 + threadIdx.x];
    double acc[HP2M_MAXJ][8];
#pragma unroll
    for (int jj = 0; jj < HP2M_MAXJ; jj++)
#pragma unroll
        for (int m = 0; m < 8; m++) acc[jj][m] = 0.0;
    __syncthreads();
    const int b = ibeg[node], mcount = numpar[node];
    for (int c0 = 0; c0 < mcount; c0 += HP2M_CHUNK) {
        int cm = min(HP2M_CHUNK, mcount - c0);
        for (int w = threadIdx.x; w < cm * 3; w += blockDim.x) {
            int i = w / 3, a = w % 3;
            const double *src = a == 0 ? sx : a == 1 ? sy : sz;
            double A[MAXNP], B[MAXNP];
            hermite_basis(n, nodes + a * np1, src[b + c0 + i], wws, len[a], A, B);
            for (int k = 0; k <= n; k++) { Ab[i][a][k] = A[k]; Bb[i][a][k] = B[k]; }
            if (a == 0) qs[i] = sq[b + c0 + i];
        }
        __syncthreads();
#pragma unroll
        for (int jj = 0; jj < HP2M_MAXJ; jj++) {
            int j = threadIdx.x + jj * HP2M_THREADS;
            if (j < P) {
                int k1 = j % np1, k2 = (j / np1) % np1, k3 = j / (np1 * np1);
                for (int i = 0; i < cm; i++) {
                    double ax = Ab[i][0][k1], bx = Bb[i][0][k1];
                    double ay = Ab[i][1][k2], by = Bb[i][1][k2];
                    double az = Ab[i][2][k3] * qs[i], bz = Bb[i][2][k3] * qs[i];
                    double axay = ax * ay, bxay = bx * ay, axby = ax * by, bxby = bx * by;
                    acc[jj][0] += axay * az;
                    acc[jj][1] += bxay * az;
                    acc[jj][2] += axby * az;
                    acc[jj][3] += axay * bz;
                    acc[jj][4] += bxby * az;
                    acc[jj][5] += axby * bz;
                    acc[jj][6] += bxay * bz;
                    acc[jj][7] += bxby * bz;
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int jj = 0; jj < HP2M_MAXJ; jj++) {
        int j = threadIdx.x + jj * HP2M_THREADS;
        if (j < P)
#pragma unroll
            for (int m = 0; m < 8; m++) Q[((size_t)node * 8 + m) * P + j] = acc[jj][m];
    }
}

// Hermite P2M over particle chunks: every node's particles are split into
// chunks of HC_PARTICLES, one block per chunk, so the root's N particles
// spread over N / HC_PARTICLES blocks instead of one.  A chunk of a node with
// a single chunk writes Q directly; the chunks of a larger node write partial
// moments that k_hermite_reduce sums in chunk order (deterministic).
// Separable form for degree <= 7: each thread owns one (k2,k3) column with
// all 8 moments x (n+1) k1 entries in registers; per particle it forms the
// four y-z products (value/derivative on each axis) times q, then 8 FMAs per
// k1 against x values every thread reads from the same shared address.
constexpr int HC_PARTICLES = 2048;
constexpr int HC_SUB = 32;

template <int NP1>
__global__ void __launch_bounds__(64)
k_p2m_hermite_sep(const HermChunk *__restrict__ chunks, const double *__restrict__ grid,
                  const double *__restrict__ box_len, const double *__restrict__ ww, const double *__restrict__ sx,
                  const double *__restrict__ sy, const double *__restrict__ sz, const double *__restrict__ sq,
                  double *__restrict__ Q, double *__restrict__ partial)
{
    constexpr int n = NP1 - 1, COLS = NP1 * NP1, P = COLS * NP1;
    const HermChunk ch = chunks[blockIdx.x];
    const int node = ch.node;
    __shared__ double nodes[3 * NP1], wws[NP1], len[3];
    __shared__ double A[3][HC_SUB][NP1], Bd[3][HC_SUB][NP1], qs[HC_SUB];
    for (int i = threadIdx.x; i < 3 * NP1; i += blockDim.x) nodes[i] = grid[(size_t)node * 3 * NP1 + i];
    for (int i = threadIdx.x; i < NP1; i += blockDim.x) wws[i] = ww[i];
    if (threadIdx.x < 3) len[threadIdx.x] = box_len[node * 3 + threadIdx.x];
    const int col = threadIdx.x;
    const bool on = col < COLS;
    const int k2 = on ? col % NP1 : 0, k3 = on ? col / NP1 : 0;
    double acc[8][NP1];
#pragma unroll
    for (int m = 0; m < 8; m++)
#pragma unroll
        for (int k = 0; k < NP1; k++) acc[m][k] = 0.0;
    __syncthreads();
    for (int c0 = 0; c0 < ch.count; c0 += HC_SUB) {
        const int cm = min(HC_SUB, ch.count - c0);
        for (int w = threadIdx.x; w < cm * 3; w += blockDim.x) {
            const int i = w / 3, ax = w % 3;
            const double *src = ax == 0 ? sx : ax == 1 ? sy : sz;
            double a[MAXNP], bb[MAXNP];
            hermite_basis(n, nodes + ax * NP1, src[ch.begin + c0 + i], wws, len[ax], a, bb);
#pragma unroll
            for (int k = 0; k < NP1; k++) { A[ax][i][k] = a[k]; Bd[ax][i][k] = bb[k]; }
            if (ax == 0) qs[i] = sq[ch.begin + c0 + i];
        }
        __syncthreads();
        for (int i = 0; i < cm; i++) {
            const double q = qs[i];
            const double az = A[2][i][k3] * q, bz = Bd[2][i][k3] * q;
            const double ay = A[1][i][k2], by = Bd[1][i][k2];
            const double yAA = ay * az, yBA = by * az, yAB = ay * bz, yBB = by * bz;
#pragma unroll
            for (int k = 0; k < NP1; k++) {
                const double ax = A[0][i][k], bx = Bd[0][i][k];
                acc[0][k] = fma(ax, yAA, acc[0][k]);
                acc[1][k] = fma(bx, yAA, acc[1][k]);
                acc[2][k] = fma(ax, yBA, acc[2][k]);
                acc[3][k] = fma(ax, yAB, acc[3][k]);
                acc[4][k] = fma(bx, yBA, acc[4][k]);
                acc[5][k] = fma(ax, yBB, acc[5][k]);
                acc[6][k] = fma(bx, yAB, acc[6][k]);
                acc[7][k] = fma(bx, yBB, acc[7][k]);
            }
        }
        __syncthreads();
    }
    if (!on) return;
    double *dst = ch.slot < 0 ? Q + (size_t)node * 8 * P : partial + (size_t)ch.slot * 8 * P;
#pragma unroll
    for (int m = 0; m < 8; m++)
#pragma unroll
        for (int k = 0; k < NP1; k++) dst[(size_t)m * P + k + NP1 * col] = acc[m][k];
}

// Degrees above 7: one thread per grid point with 8 accumulators, over the
// same chunks.
__global__ void __launch_bounds__(HP2M_THREADS)
k_p2m_hermite_chunks(int n, const HermChunk *__restrict__ chunks, const double *__restrict__ grid,
                     const double *__restrict__ box_len, const double *__restrict__ ww,
                     const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ sz,
                     const double *__restrict__ sq, double *__restrict__ Q, double *__restrict__ partial)
{
    const HermChunk ch = chunks[blockIdx.x];
    const int node = ch.node;
    const int np1 = n + 1, P = np1 * np1 * np1;
    __shared__ double nodes[3 * MAXNP], wws[MAXNP], len[3];
    __shared__ double Ab[HP2M_CHUNK][3][MAXNP], Bb[HP2M_CHUNK][3][MAXNP];
    __shared__ double qs[HP2M_CHUNK];
    for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) nodes[i] = grid[(size_t)node * 3 * np1 + i];
    for (int i = threadIdx.x; i < np1; i += blockDim.x) wws[i] = ww[i];
    if (threadIdx.x < 3) len[threadIdx.x] = box_len[node * 3 + threadIdx.x];
    double acc[HP2M_MAXJ][8];
#pragma unroll
    for (int jj = 0; jj < HP2M_MAXJ; jj++)
#pragma unroll
        for (int m = 0; m < 8; m++) acc[jj][m] = 0.0;
    __syncthreads();
    for (int c0 = 0; c0 < ch.count; c0 += HP2M_CHUNK) {
        int cm = min(HP2M_CHUNK, ch.count - c0);
        for (int w = threadIdx.x; w < cm * 3; w += blockDim.x) {
            int i = w / 3, a = w % 3;
            const double *src = a == 0 ? sx : a == 1 ? sy : sz;
            double A[MAXNP], B[MAXNP];
            hermite_basis(n, nodes + a * np1, src[ch.begin + c0 + i], wws, len[a], A, B);
            for (int k = 0; k <= n; k++) { Ab[i][a][k] = A[k]; Bb[i][a][k] = B[k]; }
            if (a == 0) qs[i] = sq[ch.begin + c0 + i];
        }
        __syncthreads();
#pragma unroll
        for (int jj = 0; jj < HP2M_MAXJ; jj++) {
            int j = threadIdx.x + jj * HP2M_THREADS;
            if (j < P) {
                int k1 = j % np1, k2 = (j / np1) % np1, k3 = j / (np1 * np1);
                for (int i = 0; i < cm; i++) {
                    double ax = Ab[i][0][k1], bx = Bb[i][0][k1];
                    double ay = Ab[i][1][k2], by = Bb[i][1][k2];
                    double az = Ab[i][2][k3] * qs[i], bz = Bb[i][2][k3] * qs[i];
                    double axay = ax * ay, bxay = bx * ay, axby = ax * by, bxby = bx * by;
                    acc[jj][0] += axay * az;
                    acc[jj][1] += bxay * az;
                    acc[jj][2] += axby * az;
                    acc[jj][3] += axay * bz;
                    acc[jj][4] += bxby * az;
                    acc[jj][5] += axby * bz;
                    acc[jj][6] += bxay * bz;
                    acc[jj][7] += bxby * bz;
                }
            }
        }
        __syncthreads();
    }
    double *dst = ch.slot < 0 ? Q + (size_t)node * 8 * P : partial + (size_t)ch.slot * 8 * P;
#pragma unroll
    for (int jj = 0; jj < HP2M_MAXJ; jj++) {
        int j = threadIdx.x + jj * HP2M_THREADS;
        if (j < P)
#pragma unroll
            for (int m = 0; m < 8; m++) dst[(size_t)m * P + j] = acc[jj][m];
    }
}

// Q of a node with several chunks = the sum of its chunks' partial moments,
// in chunk order.  red[r] = (node, first slot, number of slots).
__global__ void k_hermite_reduce(int width, const int3 *__restrict__ red, const double *__restrict__ partial,
                                 double *__restrict__ Q)
{
    const int3 r = red[blockIdx.y];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < width; j += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < r.z; c++) s += partial[(size_t)(r.y + c) * width + j];
        Q[(size_t)r.x * width + j] = s;
    }
}

int hermite_chunks(int nnodes, const int *ibeg, const int *numpar, std::vector<HermChunk> &chunks,
                   std::vector<int3> &red)
{
    chunks.clear();
    red.clear();
    int slots = 0;
    for (int v = 0; v < nnodes; v++) {
        const int np = numpar[v], nc = (np + HC_PARTICLES - 1) / HC_PARTICLES;
        if (nc <= 1) {
            chunks.push_back(HermChunk{v, ibeg[v], np, -1});
            continue;
        }
        red.push_back(make_int3(v, slots, nc));
        for (int c = 0; c < nc; c++)
            chunks.push_back(HermChunk{v, ibeg[v] + c * HC_PARTICLES, std::min(HC_PARTICLES, np - c * HC_PARTICLES),
                                       slots++});
    }
    return slots;
}

void launch_p2m_hermite(int n, int nchunks, const HermChunk *chunks, int nred, const int3 *red, const double *grid,
                        const double *box_len, const double *ww, const double *sx, const double *sy, const double *sz,
                        const double *sq, double *Q, double *partial, cudaStream_t st)
{
    if (nchunks <= 0) return;
    switch (n + 1) {
#define BT_HC(N) case N: k_p2m_hermite_sep<N><<<nchunks, 64, 0, st>>>(chunks, grid, box_len, ww, sx, sy, sz, sq, Q, partial); break;
        BT_HC(2) BT_HC(3) BT_HC(4) BT_HC(5) BT_HC(6) BT_HC(7) BT_HC(8)
#undef BT_HC
    default:
        k_p2m_hermite_chunks<<<nchunks, HP2M_THREADS, 0, st>>>(n, chunks, grid, box_len, ww, sx, sy, sz, sq, Q, partial);
    }
    launch_hermite_reduce(n, nred, red, partial, Q, st);
}

void launch_hermite_reduce(int n, int nred, const int3 *red, const double *partial, double *Q, cudaStream_t st)
{
    if (nred > 0) {
        const int width = 8 * (n + 1) * (n + 1) * (n + 1);
        dim3 g((width + 255) / 256, nred);
        k_hermite_reduce<<<g, 256, 0, st>>>(width, red, partial, Q);
    }
}

// ---------------------------------------------------------------------------
// Particle-output evaluation: PC (clusters) + PP (particles) per target leaf.
// One CTA per work item (target leaf, chunk of TB * EV_THREADS targets), TB
// targets per thread (ti and ti + EV_THREADS, ...) so that every grid point
// or source read from shared memory serves TB evaluations; FP64 accumulation
// in registers in each target's own order (the same order for any TB);
// exactly one writer per target.  TB = 2 where the work items fill the GPU
// several times over, else 1 (fp64_targets_per_thread).
// ---------------------------------------------------------------------------
constexpr int EV_THREADS = 128;
constexpr int PP_TILE = 512;

template <int KT, bool HERM, int EV_TB>
__global__ void __launch_bounds__(EV_THREADS)
k_eval_targets(int n, const int2 *__restrict__ items, const int *__restrict__ leaf_node,
               const int *__restrict__ t_ibeg, const int *__restrict__ t_numpar,
               const int64_t *__restrict__ a_off, const int *__restrict__ a_idx,
               const int64_t *__restrict__ d_off, const int *__restrict__ d_idx,
               const int *__restrict__ s_ibeg, const int *__restrict__ s_numpar, const double *__restrict__ s_grid,
               const double *__restrict__ Q, const double *__restrict__ sx, const double *__restrict__ sy,
               const double *__restrict__ sz, const double *__restrict__ sq,
               const double *__restrict__ tx, const double *__restrict__ ty, const double *__restrict__ tz,
               double kp, double kp2, double *__restrict__ pot)
{
    extern __shared__ double sm[];
    const int2 it = items[blockIdx.x];
    const int u = it.x;
    const int tnode = leaf_node[u];
    const int tb = t_ibeg[tnode], tn = t_numpar[tnode];
    bool active[EV_TB];
    int t[EV_TB];
    double x[EV_TB], y[EV_TB], z[EV_TB], acc[EV_TB];
#pragma unroll
    for (int b = 0; b < EV_TB; b++) {
        const int ti = it.y * (EV_TB * EV_THREADS) + b * EV_THREADS + threadIdx.x;
        active[b] = ti < tn;
        t[b] = tb + (active[b] ? ti : 0);
        x[b] = tx[t[b]]; y[b] = ty[t[b]]; z[b] = tz[t[b]];
        acc[b] = 0.0;
    }
    const bool any = active[0];     // target b > 0 is active only if target 0 is
    const int np1 = n + 1, P = np1 * np1 * np1;

    // far field: source clusters
    for (int64_t e = a_off[u]; e < a_off[u + 1]; e++) {
        const int s = a_idx[e];
        double *g = sm;
        double *q = sm + 3 * np1;
        const int nq = HERM ? 8 * P : P;
        const double *Qs = Q + (size_t)s * nq;
        for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) g[i] = s_grid[(size_t)s * 3 * np1 + i];
        for (int i = threadIdx.x; i < nq; i += blockDim.x) q[i] = Qs[i];
        __syncthreads();
        if (any) {
            int j = 0;
            for (int k3 = 0; k3 < np1; k3++) {
                const double gz = g[2 * np1 + k3];
                for (int k2 = 0; k2 < np1; k2++) {
                    const double gy = g[np1 + k2];
                    if (!HERM && KT <= K_REGCOULOMB) {
                        double dyz[EV_TB];
#pragma unroll
                        for (int b = 0; b < EV_TB; b++) {
                            const double dz = z[b] - gz, dy = y[b] - gy;
                            dyz[b] = dy * dy + dz * dz;
                        }
                        for (int k1 = 0; k1 < np1; k1++, j++) {
                            const double gx = g[k1], qj = q[j];
#pragma unroll
                            for (int b = 0; b < EV_TB; b++) {
                                const double dx = x[b] - gx;
                                acc[b] += k_far<KT>(fma(dx, dx, dyz[b]), qj, kp);
                            }
                        }
                    } else if (!HERM) {
                        for (int k1 = 0; k1 < np1; k1++, j++) {
#pragma unroll
                            for (int b = 0; b < EV_TB; b++)
                                acc[b] += k_any<KT, false>(x[b] - g[k1], y[b] - gy, z[b] - gz, q[j], kp, kp2);
                        }
                    } else {
                        for (int k1 = 0; k1 < np1; k1++, j++) {
#pragma unroll
                            for (int b = 0; b < EV_TB; b++)
                                acc[b] += k_pc_herm<KT>(x[b] - g[k1], y[b] - gy, z[b] - gz, q + j, P, kp);
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    // near field: source particles
    double4 *tile = reinterpret_cast<double4 *>(sm);
    for (int64_t e = d_off[u]; e < d_off[u + 1]; e++) {
        const int s = d_idx[e];
        const int sb = s_ibeg[s], sn = s_numpar[s];
        for (int c0 = 0; c0 < sn; c0 += PP_TILE) {
            int cm = min(PP_TILE, sn - c0);
            for (int i = threadIdx.x; i < cm; i += blockDim.x)
                tile[i] = make_double4(sx[sb + c0 + i], sy[sb + c0 + i], sz[sb + c0 + i], sq[sb + c0 + i]);
            __syncthreads();
            if (any) {
                for (int i = 0; i < cm; i++) {
                    const double4 p = tile[i];
#pragma unroll
                    for (int b = 0; b < EV_TB; b++)
                        acc[b] += k_any<KT, true>(x[b] - p.x, y[b] - p.y, z[b] - p.z, p.w, kp, kp2);
                }
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int b = 0; b < EV_TB; b++)
        if (active[b]) pot[t[b]] = acc[b];
}

int fp64_targets_chunk(int tb) { return tb * EV_THREADS; }

int fp64_targets_per_thread(int nunits, const int *count)
{
    // work items of two targets per thread; under about four waves of
    // resident blocks (16 blocks of 128 threads on each of ~148 SMs) one
    // target per thread keeps twice as many blocks in flight
    long long items = 0;
    for (int u = 0; u < nunits; u++) items += (count[u] + 2 * EV_THREADS - 1) / (2 * EV_THREADS);
    return items >= 4LL * 16 * 148 ? 2 : 1;
}

// ---------------------------------------------------------------------------
// Grid-output evaluation: M2L (source clusters, CC) + CP (source particles)
// onto the grid of a target node.  One thread per target grid point.
// ---------------------------------------------------------------------------
template <int KT, bool HERM>
__global__ void __launch_bounds__(EV_THREADS)
k_eval_grids(int n, const int2 *__restrict__ items, const double *__restrict__ t_grid,
             const int64_t *__restrict__ c_off, const int *__restrict__ c_idx,
             const int64_t *__restrict__ p_off, const int *__restrict__ p_idx,
             const int *__restrict__ s_ibeg, const int *__restrict__ s_numpar, const double *__restrict__ s_grid,
             const double *__restrict__ Q, const double *__restrict__ sx, const double *__restrict__ sy,
             const double *__restrict__ sz, const double *__restrict__ sq, double kp, double kp2,
             double *__restrict__ Phi)
{
    extern __shared__ double sm[];
    const int2 it = items[blockIdx.x];
    const int T = it.x;
    const int np1 = n + 1, P = np1 * np1 * np1;
    const int j0 = it.y * EV_THREADS + threadIdx.x;
    const bool active = j0 < P;
    const int jj = active ? j0 : 0;
    const double *tg = t_grid + (size_t)T * 3 * np1;
    const double x = tg[jj % np1], y = tg[np1 + (jj / np1) % np1], z = tg[2 * np1 + jj / (np1 * np1)];
    double acc[HERM ? 8 : 1];
#pragma unroll
    for (int m = 0; m < (HERM ? 8 : 1); m++) acc[m] = 0.0;

    if (!HERM) {
        for (int64_t e = c_off[T]; e < c_off[T + 1]; e++) {
            const int s = c_idx[e];
            double *g = sm;
            double *q = sm + 3 * np1;
            for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) g[i] = s_grid[(size_t)s * 3 * np1 + i];
            for (int i = threadIdx.x; i < P; i += blockDim.x) q[i] = Q[(size_t)s * P + i];
            __syncthreads();
            if (active) {
                int j = 0;
                for (int k3 = 0; k3 < np1; k3++) {
                    double dz = z - g[2 * np1 + k3];
                    for (int k2 = 0; k2 < np1; k2++) {
                        double dy = y - g[np1 + k2];
                        if (KT <= K_REGCOULOMB) {
                            double dyz = dy * dy + dz * dz;
                            for (int k1 = 0; k1 < np1; k1++, j++) {
                                double dx = x - g[k1];
                                acc[0] += k_far<KT>(fma(dx, dx, dyz), q[j], kp);
                            }
                        } else {
                            for (int k1 = 0; k1 < np1; k1++, j++)
                                acc[0] += k_any<KT, false>(x - g[k1], dy, dz, q[j], kp, kp2);
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    double4 *tile = reinterpret_cast<double4 *>(sm);
    for (int64_t e = p_off[T]; e < p_off[T + 1]; e++) {
        const int s = p_idx[e];
        const int sb = s_ibeg[s], sn = s_numpar[s];
        for (int c0 = 0; c0 < sn; c0 += PP_TILE) {
            int cm = min(PP_TILE, sn - c0);
            for (int i = threadIdx.x; i < cm; i += blockDim.x)
                tile[i] = make_double4(sx[sb + c0 + i], sy[sb + c0 + i], sz[sb + c0 + i], sq[sb + c0 + i]);
            __syncthreads();
            if (active) {
                for (int i = 0; i < cm; i++) {
                    double4 p = tile[i];
                    if (!HERM) {
                        acc[0] += k_any<KT, false>(x - p.x, y - p.y, z - p.z, p.w, kp, kp2);
                    } else {
                        k_cp_herm<KT>(p.x - x, p.y - y, p.z - z, p.w, kp, acc);
                    }
                }
            }
            __syncthreads();
        }
    }
    if (active) {
        if (!HERM) Phi[(size_t)T * P + j0] = acc[0];
        else
#pragma unroll
            for (int m = 0; m < 8; m++) Phi[((size_t)T * 8 + m) * P + j0] = acc[m];
    }
}

// ---------------------------------------------------------------------------
// Downward pass to particles
// ---------------------------------------------------------------------------

// L2P at target leaves (cp_comp_pot, src/interaction_compute/interaction_compute_downpass.c:326-497):
// pot[t] += sum_k Lx_t[k1] Ly_t[k2] Lz_t[k3] Phi[leaf][k].
constexpr int L2P_THREADS = 128;

__global__ void __launch_bounds__(L2P_THREADS)
k_l2p(int n, const int2 *__restrict__ items, const int *__restrict__ leaf_node, const int *__restrict__ t_ibeg,
      const int *__restrict__ t_numpar, const double *__restrict__ t_grid, const double *__restrict__ Phi,
      const double *__restrict__ tx, const double *__restrict__ ty, const double *__restrict__ tz,
      const double *__restrict__ mult, double *__restrict__ pot)
{
    extern __shared__ double sm[];
    const int2 it = items[blockIdx.x];
    const int node = leaf_node[it.x];
    const int np1 = n + 1, P = np1 * np1 * np1;
    double *g = sm, *ph = sm + 3 * np1;
    double *Lb = ph + P;   // [3][np1][L2P_THREADS]
    for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) g[i] = t_grid[(size_t)node * 3 * np1 + i];
    for (int i = threadIdx.x; i < P; i += blockDim.x) ph[i] = Phi[(size_t)node * P + i];
    __syncthreads();
    const int ti = it.y * L2P_THREADS + threadIdx.x;
    if (ti >= t_numpar[node]) return;
    const int t = t_ibeg[node] + ti;
    const double c[3] = {tx[t], ty[t], tz[t]};
    for (int a = 0; a < 3; a++) {
        double L[MAXNP];
        lagrange_basis(n, g + a * np1, c[a], L);
        for (int k = 0; k <= n; k++) Lb[(a * np1 + k) * L2P_THREADS + threadIdx.x] = L[k];
    }
    double acc = 0.0;
    int j = 0;
    for (int k3 = 0; k3 < np1; k3++) {
        double s3 = 0.0;
        for (int k2 = 0; k2 < np1; k2++) {
            double s2 = 0.0;
            for (int k1 = 0; k1 < np1; k1++, j++) s2 += Lb[(0 * np1 + k1) * L2P_THREADS + threadIdx.x] * ph[j];
            s3 += Lb[(1 * np1 + k2) * L2P_THREADS + threadIdx.x] * s2;
        }
        acc += Lb[(2 * np1 + k3) * L2P_THREADS + threadIdx.x] * s3;
    }
    pot[t] += mult ? -mult[t] * acc : acc;
}

// Hermite downward pass (cp_comp_pot_hermite, src/interaction_compute/interaction_compute_downpass.c:860-1109):
// every target node interpolates its 8 grid arrays to its own targets; here
// each target leaf gathers from itself and all its ancestors, so each target
// has one writer.
__global__ void __launch_bounds__(L2P_THREADS)
k_l2p_hermite(int n, const int2 *__restrict__ items, const int *__restrict__ leaf_node,
              const int *__restrict__ parent, const int *__restrict__ t_ibeg, const int *__restrict__ t_numpar,
              const double *__restrict__ t_grid, const double *__restrict__ box_len, const double *__restrict__ ww,
              const double *__restrict__ Phi, const double *__restrict__ tx, const double *__restrict__ ty,
              const double *__restrict__ tz, double *__restrict__ pot)
{
    extern __shared__ double sm[];
    const int2 it = items[blockIdx.x];
    const int leaf = leaf_node[it.x];
    const int np1 = n + 1, P = np1 * np1 * np1;
    double *g = sm, *ph = sm + 3 * np1;                 // ph: 8*P
    double *AB = ph + 8 * P;                             // [6][np1][L2P_THREADS]
    __shared__ double wws[MAXNP], len[3];
    for (int i = threadIdx.x; i < np1; i += blockDim.x) wws[i] = ww[i];
    const int ti = it.y * L2P_THREADS + threadIdx.x;
    const bool active = ti < t_numpar[leaf];
    const int t = t_ibeg[leaf] + (active ? ti : 0);
    const double c[3] = {tx[t], ty[t], tz[t]};
    double acc = 0.0;
    for (int node = leaf; node >= 0; node = parent[node]) {
        __syncthreads();
        for (int i = threadIdx.x; i < 3 * np1; i += blockDim.x) g[i] = t_grid[(size_t)node * 3 * np1 + i];
        for (int i = threadIdx.x; i < 8 * P; i += blockDim.x) ph[i] = Phi[(size_t)node * 8 * P + i];
        if (threadIdx.x < 3) len[threadIdx.x] = box_len[node * 3 + threadIdx.x];
        __syncthreads();
        if (!active) continue;
        for (int a = 0; a < 3; a++) {
            double A[MAXNP], B[MAXNP];
            hermite_basis(n, g + a * np1, c[a], wws, len[a], A, B);
            for (int k = 0; k <= n; k++) {
                AB[((2 * a) * np1 + k) * L2P_THREADS + threadIdx.x] = A[k];
                AB[((2 * a + 1) * np1 + k) * L2P_THREADS + threadIdx.x] = B[k];
            }
        }
#define AX(k) AB[((0) * np1 + (k)) * L2P_THREADS + threadIdx.x]
#define BX(k) AB[((1) * np1 + (k)) * L2P_THREADS + threadIdx.x]
#define AY(k) AB[((2) * np1 + (k)) * L2P_THREADS + threadIdx.x]
#define BY(k) AB[((3) * np1 + (k)) * L2P_THREADS + threadIdx.x]
#define AZ(k) AB[((4) * np1 + (k)) * L2P_THREADS + threadIdx.x]
#define BZ(k) AB[((5) * np1 + (k)) * L2P_THREADS + threadIdx.x]
        int j = 0;
        for (int k3 = 0; k3 < np1; k3++) {
            double az = AZ(k3), bz = BZ(k3);
            for (int k2 = 0; k2 < np1; k2++) {
                double ay = AY(k2), by = BY(k2);
                for (int k1 = 0; k1 < np1; k1++, j++) {
                    double ax = AX(k1), bx = BX(k1);
                    acc += ax * ay * az * ph[j] + bx * ay * az * ph[P + j] + ax * by * az * ph[2 * P + j]
                         + ax * ay * bz * ph[3 * P + j] + bx * by * az * ph[4 * P + j]
                         + ax * by * bz * ph[5 * P + j] + bx * ay * bz * ph[6 * P + j]
                         + bx * by * bz * ph[7 * P + j];
                }
            }
        }
#undef AX
#undef BX
#undef AY
#undef BY
#undef AZ
#undef BZ
    }
    if (active) pot[t] += acc;
}

// ---------------------------------------------------------------------------
// FP64 direct sum (InteractionCompute_Direct, src/interaction_compute/interaction_compute_direct.c:26-231)
// ---------------------------------------------------------------------------
template <int KT>
__global__ void __launch_bounds__(EV_THREADS)
k_direct(int nt, int ns, const double *__restrict__ tx, const double *__restrict__ ty, const double *__restrict__ tz,
         const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ sz,
         const double *__restrict__ sq, double kp, double kp2, double *__restrict__ out)
{
    __shared__ double4 tile[PP_TILE];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = t < nt;
    const double x = active ? tx[t] : 0.0, y = active ? ty[t] : 0.0, z = active ? tz[t] : 0.0;
    double acc = 0.0;
    for (int c0 = 0; c0 < ns; c0 += PP_TILE) {
        int cm = min(PP_TILE, ns - c0);
        for (int i = threadIdx.x; i < cm; i += blockDim.x)
            tile[i] = make_double4(sx[c0 + i], sy[c0 + i], sz[c0 + i], sq[c0 + i]);
        __syncthreads();
        for (int i = 0; i < cm; i++) {
            double4 p = tile[i];
            acc += k_any<KT, true>(x - p.x, y - p.y, z - p.z, p.w, kp, kp2);
        }
        __syncthreads();
    }
    if (active) out[t] = acc;
}

// Output in the caller's order (Particles_Targets_Reorder, src/particles/particles.c:58-94).
__global__ void k_scatter(int n, const int *__restrict__ order, const double *__restrict__ src, double *__restrict__ dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[order[i]] = src[i];
}

// Throughput probes: independent FMA chains per thread (8 in flight), and a
// reciprocal-square-root stream.  The results are written so nothing is dead.
template <typename R>
__global__ void k_fma_probe(int iters, R seed, R *out)
{
    R a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + (R)(threadIdx.x + k);
    const R b = (R)0.9999999, c = (R)1e-7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = a[k] * b + c;
    }
    R s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == (R)-1) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_rsqrt_probe(int iters, float seed, float *out)
{
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + (float)(threadIdx.x + k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = rsqrtf(a[k]);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == -1.f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

void launch_scatter(int n, const int *order, const double *src, double *dst, cudaStream_t st)
{
    if (n > 0) k_scatter<<<(n + 255) / 256, 256, 0, st>>>(n, order, src, dst);
}

__global__ void k_gather(int n, const int *__restrict__ order, const double *__restrict__ src, double *__restrict__ dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[order[i]];
}

void launch_gather(int n, const int *order, const double *src, double *dst, cudaStream_t st)
{
    if (n > 0) k_gather<<<(n + 255) / 256, 256, 0, st>>>(n, order, src, dst);
}

// Returns device milliseconds of one probe launch; ops = launched FMA/rsqrt count.
float run_probe(int which, int sms, double *ops, void *scratch, cudaStream_t st)
{
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sms * 8, threads = 256, iters = 4096;
    for (int rep = 0; rep < 2; rep++) {
        cudaEventRecord(a, st);
        if (which == 0) k_fma_probe<double><<<blocks, threads, 0, st>>>(iters, 1.0, (double *)scratch);
        else if (which == 1) k_fma_probe<float><<<blocks, threads, 0, st>>>(iters, 1.0f, (float *)scratch);
        else k_rsqrt_probe<<<blocks, threads, 0, st>>>(iters, 2.0f, (float *)scratch);
        cudaEventRecord(b, st);
    }
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ops = (double)blocks * threads * iters * 8;
    return ms;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static size_t kron_smem(int n)
{
    int np1 = n + 1, P = np1 * np1 * np1;
    return sizeof(double) * (size_t)(3 * np1 * np1 + 4 * P);
}

void launch_p2m(int n, bool hermite, int nleaves, const int *leaves, int nnodes, const int *ibeg, const int *numpar,
                const double *grid, const double *box_len, const double *ww, const double *sx, const double *sy,
                const double *sz, const double *sq, double *Q, cudaStream_t st)
{
    if (!hermite) {
        if (nleaves <= 0) return;
        switch (n + 1) {
#define BT_P2S(N) case N: k_p2m_sep<N><<<nleaves, P2S_THREADS, 0, st>>>(leaves, ibeg, numpar, grid, sx, sy, sz, sq, Q); return;
            BT_P2S(2) BT_P2S(3) BT_P2S(4) BT_P2S(5) BT_P2S(6) BT_P2S(7) BT_P2S(8)
            BT_P2S(9) BT_P2S(10) BT_P2S(11) BT_P2S(12) BT_P2S(13)
#undef BT_P2S
        }
        k_p2m_lagrange<<<nleaves, P2M_THREADS, 0, st>>>(n, leaves, ibeg, numpar, grid, sx, sy, sz, sq, Q);
    } else {
        if (nnodes > 0)
            k_p2m_hermite<<<nnodes, HP2M_THREADS, 0, st>>>(n, ibeg, numpar, grid, box_len, ww, sx, sy, sz, sq, Q);
    }
}

void launch_m2m(int n, int nparents, const int *parents, const int *nchild, const int *child, const double *grid,
                double *Q, cudaStream_t st)
{
    if (nparents <= 0) return;
    size_t sm = kron_smem(n);
    cudaFuncSetAttribute(k_m2m, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_m2m<<<nparents, 256, sm, st>>>(n, parents, nchild, child, grid, Q);
}

void launch_l2l(int n, int nparents, const int *parents, const int *nchild, const int *child, const double *grid,
                double *Phi, cudaStream_t st)
{
    if (nparents <= 0) return;
    size_t sm = kron_smem(n);
    cudaFuncSetAttribute(k_l2l, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_l2l<<<nparents, 256, sm, st>>>(n, parents, nchild, child, grid, Phi);
}

template <int KT, bool HERM>
static void eval_targets_t(const EvalTargetsArgs &a, cudaStream_t st)
{
    int np1 = a.n + 1, P = np1 * np1 * np1;
    size_t far = sizeof(double) * (size_t)(3 * np1 + (HERM ? 8 * P : P));
    size_t near = sizeof(double4) * PP_TILE;
    size_t sm = far > near ? far : near;
    auto fn = a.tb == 2 ? k_eval_targets<KT, HERM, 2> : k_eval_targets<KT, HERM, 1>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    fn<<<a.nitems, EV_THREADS, sm, st>>>(a.n, a.items, a.leaf_node, a.t_ibeg, a.t_numpar, a.a_off, a.a_idx,
                                         a.d_off, a.d_idx, a.s_ibeg, a.s_numpar, a.s_grid, a.Q, a.sx, a.sy,
                                         a.sz, a.sq, a.tx, a.ty, a.tz, a.kp, a.kp2, a.pot);
}

// Kernels with Hermite forms: Coulomb, Yukawa, regularized Coulomb, sin-over-r.
void launch_eval_targets(int kernel, bool hermite, const EvalTargetsArgs &a, cudaStream_t st)
{
    if (a.nitems <= 0) return;
    switch (kernel) {
    case K_COULOMB: hermite ? eval_targets_t<K_COULOMB, true>(a, st) : eval_targets_t<K_COULOMB, false>(a, st); break;
    case K_YUKAWA: hermite ? eval_targets_t<K_YUKAWA, true>(a, st) : eval_targets_t<K_YUKAWA, false>(a, st); break;
    case K_REGCOULOMB:
        hermite ? eval_targets_t<K_REGCOULOMB, true>(a, st) : eval_targets_t<K_REGCOULOMB, false>(a, st);
        break;
    case K_SINOVERR:
        hermite ? eval_targets_t<K_SINOVERR, true>(a, st) : eval_targets_t<K_SINOVERR, false>(a, st);
        break;
    case K_REGYUKAWA: eval_targets_t<K_REGYUKAWA, false>(a, st); break;
    case K_ATAN: eval_targets_t<K_ATAN, false>(a, st); break;
    case K_MQ: eval_targets_t<K_MQ, false>(a, st); break;
    case K_RBSU: eval_targets_t<K_RBSU, false>(a, st); break;
    case K_RBSV: eval_targets_t<K_RBSV, false>(a, st); break;
    default: eval_targets_t<K_USER, false>(a, st);
    }
}

template <int KT, bool HERM>
static void eval_grids_t(const EvalGridsArgs &a, cudaStream_t st)
{
    int np1 = a.n + 1, P = np1 * np1 * np1;
    size_t far = sizeof(double) * (size_t)(3 * np1 + P);
    size_t near = sizeof(double4) * PP_TILE;
    size_t sm = far > near ? far : near;
    auto fn = k_eval_grids<KT, HERM>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    fn<<<a.nitems, EV_THREADS, sm, st>>>(a.n, a.items, a.t_grid, a.c_off, a.c_idx, a.p_off, a.p_idx, a.s_ibeg,
                                         a.s_numpar, a.s_grid, a.Q, a.sx, a.sy, a.sz, a.sq, a.kp, a.kp2, a.Phi);
}

// Grid outputs (CP, CC) exist for all but the periodic kernels (atan, MQ).
void launch_eval_grids(int kernel, bool hermite, const EvalGridsArgs &a, cudaStream_t st)
{
    if (a.nitems <= 0) return;
    switch (kernel) {
    case K_COULOMB: hermite ? eval_grids_t<K_COULOMB, true>(a, st) : eval_grids_t<K_COULOMB, false>(a, st); break;
    case K_YUKAWA: hermite ? eval_grids_t<K_YUKAWA, true>(a, st) : eval_grids_t<K_YUKAWA, false>(a, st); break;
    case K_REGCOULOMB:
        hermite ? eval_grids_t<K_REGCOULOMB, true>(a, st) : eval_grids_t<K_REGCOULOMB, false>(a, st);
        break;
    case K_SINOVERR: hermite ? eval_grids_t<K_SINOVERR, true>(a, st) : eval_grids_t<K_SINOVERR, false>(a, st); break;
    case K_REGYUKAWA: eval_grids_t<K_REGYUKAWA, false>(a, st); break;
    case K_RBSU: eval_grids_t<K_RBSU, false>(a, st); break;
    case K_RBSV: eval_grids_t<K_RBSV, false>(a, st); break;
    default: eval_grids_t<K_USER, false>(a, st);
    }
}

void launch_l2p(int n, bool hermite, int nitems, const int2 *items, const int *leaf_node, const int *parent,
                const int *t_ibeg, const int *t_numpar, const double *t_grid, const double *box_len,
                const double *ww, const double *Phi, const double *tx, const double *ty, const double *tz,
                double *pot, cudaStream_t st, const double *mult)
{
    if (nitems <= 0) return;
    int np1 = n + 1, P = np1 * np1 * np1;
    if (!hermite) {
        size_t sm = sizeof(double) * (size_t)(3 * np1 + P + 3 * np1 * L2P_THREADS);
        cudaFuncSetAttribute(k_l2p, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_l2p<<<nitems, L2P_THREADS, sm, st>>>(n, items, leaf_node, t_ibeg, t_numpar, t_grid, Phi, tx, ty, tz, mult,
                                               pot);
    } else {
        size_t sm = sizeof(double) * (size_t)(3 * np1 + 8 * P + 6 * np1 * L2P_THREADS);
        cudaFuncSetAttribute(k_l2p_hermite, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_l2p_hermite<<<nitems, L2P_THREADS, sm, st>>>(n, items, leaf_node, parent, t_ibeg, t_numpar, t_grid,
                                                       box_len, ww, Phi, tx, ty, tz, pot);
    }
}

void launch_direct(int kernel, int nt, int ns, const double *tx, const double *ty, const double *tz,
                   const double *sx, const double *sy, const double *sz, const double *sq, double kp, double *out,
                   cudaStream_t st, double kp2)
{
    if (nt <= 0) return;
    int grid = (nt + EV_THREADS - 1) / EV_THREADS;
#define BT_DIRECT(K) k_direct<K><<<grid, EV_THREADS, 0, st>>>(nt, ns, tx, ty, tz, sx, sy, sz, sq, kp, kp2, out)
    switch (kernel) {
    case K_COULOMB: BT_DIRECT(K_COULOMB); break;
    case K_YUKAWA: BT_DIRECT(K_YUKAWA); break;
    case K_REGCOULOMB: BT_DIRECT(K_REGCOULOMB); break;
    case K_REGYUKAWA: BT_DIRECT(K_REGYUKAWA); break;
    case K_ATAN: BT_DIRECT(K_ATAN); break;
    case K_SINOVERR: BT_DIRECT(K_SINOVERR); break;
    case K_MQ: BT_DIRECT(K_MQ); break;
    case K_RBSU: BT_DIRECT(K_RBSU); break;
    case K_RBSV: BT_DIRECT(K_RBSV); break;
    default: BT_DIRECT(K_USER);
    }
#undef BT_DIRECT
}

}  // namespace bt
