// bt_learned.cu -- learned interpolation-degree selection for particle-cluster
// interactions: features, training labels made by the treecode itself, and a
// small MLP (6 -> 64 -> 64 -> 64 -> 11, tanh) with hand-written forward,
// backward and Adam kernels (FP32).
//
// Label of an interaction (target batch B, source cluster C) at degree d:
//   eta_d = RMS over sampled targets t of |phi_d(t) - phi(t)| / (||q_C||_2 / dist)
// where phi is the exact FP64 sum over C's particles, phi_d the degree-d
// barycentric approximation from C's proxy charges, and dist the distance
// between the batch and cluster centres (the MAC distance of
// src/interaction_lists/interaction_lists.c:476-486).  For charges of random
// sign the far-field terms of a target add in quadrature, so keeping every
// interaction at eta_d <= tol keeps the relative L2 error of the far field at
// or below tol.  The network predicts log10(eta_d) for d = 2..12.
#include <cuda_runtime.h>

#include <algorithm>

#include <cfloat>
#include <cstdint>

#include "bt_learned.h"

namespace bt {

// ---------------------------------------------------------------------------
// node charge moments and interaction features
// ---------------------------------------------------------------------------
// Charge moments of every node: sum |q| and sqrt(sum q^2).  Leaves sum their
// particles (one block per leaf); every other node sums its children, level
// by level from the deepest (a fixed order, so the features are the same
// bits on every call).
__global__ void k_leaf_moments(int nleaves, const int *__restrict__ leaves, const int *__restrict__ ibeg,
                               const int *__restrict__ numpar, const double *__restrict__ q, double *__restrict__ mom)
{
    const int node = leaves[blockIdx.x];
    double a = 0.0, b = 0.0;
    for (int i = ibeg[node] + threadIdx.x; i < ibeg[node] + numpar[node]; i += blockDim.x) {
        double v = q[i];
        a += fabs(v);
        b += v * v;
    }
    __shared__ double sa[256], sb[256];
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) { sa[threadIdx.x] += sa[threadIdx.x + s]; sb[threadIdx.x] += sb[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { mom[2 * node] = sa[0]; mom[2 * node + 1] = sb[0]; }
}

__global__ void k_moments_up(int cnt, const int *__restrict__ nodes, const int *__restrict__ nchild,
                             const int *__restrict__ child, double *__restrict__ mom)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cnt) return;
    const int node = nodes[k];
    double a = 0.0, b = 0.0;
    for (int c = 0; c < nchild[node]; c++) {
        const int ch = child[8 * node + c];
        a += mom[2 * ch];
        b += mom[2 * ch + 1];
    }
    mom[2 * node] = a;
    mom[2 * node + 1] = b;
}

__global__ void k_moments_sqrt(int n, double *__restrict__ mom)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) mom[2 * k + 1] = sqrt(mom[2 * k + 1]);
}

__device__ __forceinline__ void features_of(const FeatureArgs &a, int tnode, int snode, float *f)
{
    double dx = a.t_ctr[3 * tnode] - a.s_ctr[3 * snode];
    double dy = a.t_ctr[3 * tnode + 1] - a.s_ctr[3 * snode + 1];
    double dz = a.t_ctr[3 * tnode + 2] - a.s_ctr[3 * snode + 2];
    double dist = sqrt(dx * dx + dy * dy + dz * dz);
    double rs = a.s_rad[snode], rt = a.t_rad[tnode];
    double ns = a.s_numpar[snode], nt = a.t_numpar[tnode];
    double q1 = a.s_mom[2 * snode], q2 = a.s_mom[2 * snode + 1];
    f[0] = (float)log10(ns);
    f[1] = (float)log10(nt);
    f[2] = (float)((rs + rt) / dist);
    f[3] = (float)(rs / dist);
    f[4] = (float)(rt / dist);
    f[5] = (float)(q2 > 0 ? q1 / (q2 * sqrt(ns)) : 0.0);
}

// One row per (target leaf unit, approx entry): CSR walk by binary search of
// the entry index in the offsets.
__global__ void k_features(FeatureArgs a, int64_t nentries, float *__restrict__ out)
{
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= nentries) return;
    int lo = 0, hi = a.units;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (a.off[mid] <= e) lo = mid; else hi = mid;
    }
    float f[MLP_IN];
    features_of(a, a.unit_node[lo], a.idx[e], f);
    for (int k = 0; k < MLP_IN; k++) out[e * MLP_IN + k] = f[k];
}

__global__ void k_features_pairs(FeatureArgs a, int n, const int *__restrict__ tnodes, const int *__restrict__ snodes,
                                 float *__restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float f[MLP_IN];
    features_of(a, tnodes[i], snodes[i], f);
    for (int k = 0; k < MLP_IN; k++) out[(size_t)i * MLP_IN + k] = f[k];
}

// ---------------------------------------------------------------------------
// training labels: per sample, the error of every degree against the exact sum
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(LBL_TARGETS)
k_labels(LabelArgs a)
{
    const int smp = blockIdx.x;
    const int tnode = a.tnodes[smp], snode = a.snodes[smp];
    const int tb = a.t_ibeg[tnode], tn = a.t_numpar[tnode];
    const int nt = min(tn, LBL_TARGETS);
    const int ti = threadIdx.x;
    const bool active = ti < nt;
    const int t = tb + (active ? (int)((long long)ti * tn / nt) : 0);
    const double x = a.tx[t], y = a.ty[t], z = a.tz[t];
    // exact far field of the cluster's particles (FP64)
    double exact = 0.0;
    if (active) {
        const int sb = a.s_ibeg[snode], sn = a.s_numpar[snode];
        for (int i = sb; i < sb + sn; i++) {
            double dx = x - a.sx[i], dy = y - a.sy[i], dz = z - a.sz[i];
            exact += a.sq[i] * rsqrt(dx * dx + dy * dy + dz * dz);
        }
    }
    __shared__ double red[LBL_TARGETS];
    double dxc = a.t_ctr[3 * tnode] - a.s_ctr[3 * snode], dyc = a.t_ctr[3 * tnode + 1] - a.s_ctr[3 * snode + 1],
           dzc = a.t_ctr[3 * tnode + 2] - a.s_ctr[3 * snode + 2];
    const double dist = sqrt(dxc * dxc + dyc * dyc + dzc * dzc);
    const double scale = a.s_mom[2 * snode + 1] / dist;
    for (int d = MLP_DMIN; d <= MLP_DMAX; d++) {
        const int np1 = d + 1, P = np1 * np1 * np1;
        const double *g = a.grid[d] + (size_t)snode * 3 * np1;
        const double *Q = a.Q[d] + (size_t)snode * P;
        double approx = 0.0;
        if (active) {
            int j = 0;
            for (int k3 = 0; k3 < np1; k3++) {
                double dz = z - g[2 * np1 + k3];
                for (int k2 = 0; k2 < np1; k2++) {
                    double dy = y - g[np1 + k2];
                    double dyz = dy * dy + dz * dz;
                    for (int k1 = 0; k1 < np1; k1++, j++) {
                        double dx = x - g[k1];
                        approx += Q[j] * rsqrt(fma(dx, dx, dyz));
                    }
                }
            }
        }
        double e = active ? (approx - exact) * (approx - exact) : 0.0;
        red[ti] = e;
        __syncthreads();
        for (int s = LBL_TARGETS / 2; s > 0; s >>= 1) {
            if (ti < s) red[ti] += red[ti + s];
            __syncthreads();
        }
        if (ti == 0) {
            double eta = sqrt(red[0] / nt) / (scale > 0 ? scale : 1e-300);
            double l = log10(eta > 1e-14 ? eta : 1e-14);
            a.labels[(size_t)smp * MLP_OUT + (d - MLP_DMIN)] = (float)(l > 2.0 ? 2.0 : l);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// MLP: layer kernels (batch-major activations, weights [in][out])
// ---------------------------------------------------------------------------
// Normalised input, clipped to +-4 standard deviations so that interactions
// outside the training range (for instance far larger clusters) are treated
// like the most extreme ones seen in training instead of being extrapolated.
__device__ __forceinline__ float norm_input(float x, float mean, float sd)
{
    return fminf(fmaxf((x - mean) / sd, -4.f), 4.f);
}

// Y[b][o] = act(sum_i X[b][i] W[i][o] + bias[o]); act: 0 none, 1 tanh.
// The input layer first applies the stored normalisation (x - mean) / std.
__global__ void k_linear_fwd(int B, int I, int O, const float *__restrict__ X, const float *__restrict__ W,
                             const float *__restrict__ bias, const float *__restrict__ norm, int act,
                             float *__restrict__ Y)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * O) return;
    int b = idx / O, o = idx % O;
    float s = bias[o];
    for (int i = 0; i < I; i++) {
        float x = X[(size_t)b * I + i];
        if (norm) x = norm_input(x, norm[i], norm[I + i]);
        s = fmaf(x, W[i * O + o], s);
    }
    Y[idx] = act ? tanhf(s) : s;
}

// dX[b][i] = (sum_o dY[b][o] W[i][o]) * (1 - A[b][i]^2)  (A = tanh output of the layer below)
__global__ void k_linear_bwd_in(int B, int I, int O, const float *__restrict__ dY, const float *__restrict__ W,
                                const float *__restrict__ A, float *__restrict__ dX)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * I) return;
    int b = idx / I, i = idx % I;
    float s = 0.f;
    for (int o = 0; o < O; o++) s = fmaf(dY[(size_t)b * O + o], W[i * O + o], s);
    float a = A[idx];
    dX[idx] = s * (1.f - a * a);
}

// gW[i][o] = sum_b X[b][i] dY[b][o];  gb[o] = sum_b dY[b][o]  (deterministic order)
__global__ void k_linear_bwd_w(int B, int I, int O, const float *__restrict__ X, const float *__restrict__ dY,
                               const float *__restrict__ norm, float *__restrict__ gW, float *__restrict__ gb)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (I + 1) * O) return;
    int i = idx / O, o = idx % O;
    float s = 0.f;
    if (i < I) {
        for (int b = 0; b < B; b++) {
            float x = X[(size_t)b * I + i];
            if (norm) x = norm_input(x, norm[i], norm[I + i]);
            s = fmaf(x, dY[(size_t)b * O + o], s);
        }
        gW[i * O + o] = s;
    } else {
        for (int b = 0; b < B; b++) s += dY[(size_t)b * O + o];
        gb[o] = s;
    }
}

// mean-squared error over all outputs: loss partials per sample, dY = 2 (Yh - Y) / (B * O)
__global__ void k_mse(int B, int O, const float *__restrict__ Yh, const float *__restrict__ Y,
                      float *__restrict__ dY, float *__restrict__ loss_per_sample)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    float s = 0.f;
    for (int o = 0; o < O; o++) {
        float d = Yh[(size_t)b * O + o] - Y[(size_t)b * O + o];
        s += d * d;
        dY[(size_t)b * O + o] = 2.f * d / (float)(B * O);
    }
    loss_per_sample[b] = s / (float)O;
}

__global__ void k_adam(int n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gi = g[i];
    float mi = b1 * m[i] + (1.f - b1) * gi;
    float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_gather_rows(int B, int width, const int *__restrict__ rows, const float *__restrict__ src,
                              float *__restrict__ dst)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * width) return;
    int b = idx / width, k = idx % width;
    dst[idx] = src[(size_t)rows[b] * width + k];
}


// ---------------------------------------------------------------------------
// host-side drivers of the layer kernels
// ---------------------------------------------------------------------------
static inline int nb(long long n, int t) { return (int)((n + t - 1) / t); }

MlpView mlp_view(float *w)
{
    MlpView v;
    v.norm = w;
    v.W[0] = w + 2 * MLP_IN;
    v.b[0] = v.W[0] + MLP_IN * MLP_H;
    v.W[1] = v.b[0] + MLP_H;
    v.b[1] = v.W[1] + MLP_H * MLP_H;
    v.W[2] = v.b[1] + MLP_H;
    v.b[2] = v.W[2] + MLP_H * MLP_H;
    v.W[3] = v.b[2] + MLP_H;
    v.b[3] = v.W[3] + MLP_H * MLP_OUT;
    return v;
}

void mlp_forward(const float *w, int B, const float *X, float *act, float *Yh, cudaStream_t st)
{
    MlpView v = mlp_view(const_cast<float *>(w));
    float *A1 = act, *A2 = act + (size_t)B * MLP_H, *A3 = act + 2 * (size_t)B * MLP_H;
    k_linear_fwd<<<nb((long long)B * MLP_H, 256), 256, 0, st>>>(B, MLP_IN, MLP_H, X, v.W[0], v.b[0], v.norm, 1, A1);
    k_linear_fwd<<<nb((long long)B * MLP_H, 256), 256, 0, st>>>(B, MLP_H, MLP_H, A1, v.W[1], v.b[1], nullptr, 1, A2);
    k_linear_fwd<<<nb((long long)B * MLP_H, 256), 256, 0, st>>>(B, MLP_H, MLP_H, A2, v.W[2], v.b[2], nullptr, 1, A3);
    k_linear_fwd<<<nb((long long)B * MLP_OUT, 256), 256, 0, st>>>(B, MLP_H, MLP_OUT, A3, v.W[3], v.b[3], nullptr, 0, Yh);
}

// Forward + backward of the MSE loss on one batch; grad has the weight layout
// (normalisation entries get zero gradient).  act: 3*B*H, dbuf: 2*B*H + B*O, lossb: B.
void mlp_forward_backward(const float *w, int B, const float *X, const float *Y, float *act, float *Yh, float *dbuf,
                          float *lossb, float *grad, cudaStream_t st)
{
    mlp_forward(w, B, X, act, Yh, st);
    MlpView v = mlp_view(const_cast<float *>(w));
    MlpView g = mlp_view(grad);
    float *A1 = act, *A2 = act + (size_t)B * MLP_H, *A3 = act + 2 * (size_t)B * MLP_H;
    float *dO = dbuf, *dH = dbuf + (size_t)B * MLP_OUT, *dH2 = dH + (size_t)B * MLP_H;
    cudaMemsetAsync(grad, 0, sizeof(float) * 2 * MLP_IN, st);
    k_mse<<<nb(B, 256), 256, 0, st>>>(B, MLP_OUT, Yh, Y, dO, lossb);
    k_linear_bwd_w<<<nb((MLP_H + 1) * MLP_OUT, 256), 256, 0, st>>>(B, MLP_H, MLP_OUT, A3, dO, nullptr, g.W[3], g.b[3]);
    k_linear_bwd_in<<<nb((long long)B * MLP_H, 256), 256, 0, st>>>(B, MLP_H, MLP_OUT, dO, v.W[3], A3, dH);
    k_linear_bwd_w<<<nb((MLP_H + 1) * MLP_H, 256), 256, 0, st>>>(B, MLP_H, MLP_H, A2, dH, nullptr, g.W[2], g.b[2]);
    k_linear_bwd_in<<<nb((long long)B * MLP_H, 256), 256, 0, st>>>(B, MLP_H, MLP_H, dH, v.W[2], A2, dH2);
    k_linear_bwd_w<<<nb((MLP_H + 1) * MLP_H, 256), 256, 0, st>>>(B, MLP_H, MLP_H, A1, dH2, nullptr, g.W[1], g.b[1]);
    k_linear_bwd_in<<<nb((long long)B * MLP_H, 256), 256, 0, st>>>(B, MLP_H, MLP_H, dH2, v.W[1], A1, dH);
    k_linear_bwd_w<<<nb((MLP_IN + 1) * MLP_H, 256), 256, 0, st>>>(B, MLP_IN, MLP_H, X, dH, v.norm, g.W[0], g.b[0]);
}

void mlp_adam(int n, float *w, const float *g, float *m, float *v, float lr, int step, cudaStream_t st)
{
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<nb(n, 256), 256, 0, st>>>(n, w, g, m, v, lr, b1, b2, 1e-8f, c1, c2);
}

void gather_rows(int B, int width, const int *rows, const float *src, float *dst, cudaStream_t st)
{
    k_gather_rows<<<nb((long long)B * width, 256), 256, 0, st>>>(B, width, rows, src, dst);
}

int launch_node_moments(const MomentTree &t, const double *q, double *mom, cudaStream_t st)
{
    if (t.nnodes <= 0) return 0;
    int launches = 0;
    if (t.nleaves > 0) {
        k_leaf_moments<<<t.nleaves, 256, 0, st>>>(t.nleaves, t.leaves, t.ibeg, t.numpar, q, mom);
        launches++;
    }
    for (int l = t.max_depth - 1; l >= 0; l--) {
        const int cnt = t.lvl_off[l + 1] - t.lvl_off[l];
        if (cnt > 0) {
            k_moments_up<<<nb(cnt, 128), 128, 0, st>>>(cnt, t.lvl_nodes + t.lvl_off[l], t.nchild, t.child, mom);
            launches++;
        }
    }
    k_moments_sqrt<<<nb(t.nnodes, 256), 256, 0, st>>>(t.nnodes, mom);
    return launches + 1;
}

void launch_features(const FeatureArgs &a, int64_t nentries, float *out, cudaStream_t st)
{
    if (nentries > 0) k_features<<<(unsigned)((nentries + 255) / 256), 256, 0, st>>>(a, nentries, out);
}

void launch_features_pairs(const FeatureArgs &a, int n, const int *tnodes, const int *snodes, float *out,
                           cudaStream_t st)
{
    if (n > 0) k_features_pairs<<<nb(n, 256), 256, 0, st>>>(a, n, tnodes, snodes, out);
}

void launch_labels(const LabelArgs &a, int nsamples, cudaStream_t st)
{
    if (nsamples > 0) k_labels<<<nsamples, LBL_TARGETS, 0, st>>>(a);
}

// Degree selection under one absolute error share per system.  The network
// predicts e_d, log10 of an interaction's error at degree d over its scale
// |q_C|_2 / d.  Errors of different interactions add at a target roughly as
// independent terms, so if every (target, cluster entry) pair of a system
// contributes at most
//   share = c tol sqrt(sum_t phi_t^2 / sum_t N_t)
// (N_t the target's cluster entries, phi_t its potential), the system's
// relative L2 error is about c tol.  phi_t^2 is estimated per target leaf
// at two sampled targets: the near-field sum sum_j q_j^2 / r_j^2 over the
// leaf's near-field leaves within twice their radius (r floored at each
// leaf's mean particle spacing), (|q_L|_2 / d)^2 for the other near-field
// leaves and per cluster entry (|q_C|_2 / d)^2 -- the mean square potential
// of charges of either sign.  Each interaction then takes the lowest degree d with
// e_d + log10(|q_C|_2 / d) <= log10(share), or direct evaluation when no
// degree qualifies or direct is cheaper.
__global__ void k_unit_phi2_sampled(FeatureArgs a, const int *__restrict__ t_ibeg, const int64_t *__restrict__ d_off,
                                    const int *__restrict__ d_idx, const int *__restrict__ s_ibeg,
                                    const double *__restrict__ sx, const double *__restrict__ sy,
                                    const double *__restrict__ sz, const double *__restrict__ sq,
                                    const double *__restrict__ tx, const double *__restrict__ ty,
                                    const double *__restrict__ tz, double *__restrict__ unit_sums)
{
    constexpr int NS = 2;                  // sampled targets per leaf: a quarter and three quarters in
    const int u = blockIdx.x;
    const int tn = a.unit_node[u], nt = a.t_numpar[tn];
    double px[NS], py[NS], pz[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) {
        const int t = t_ibeg[tn] + (int)(((2 * k + 1) * (int64_t)nt) / (2 * NS));
        px[k] = tx[t]; py[k] = ty[t]; pz[k] = tz[t];
    }
    double phi2 = 0.0;
    for (int64_t e = a.off[u] + threadIdx.x; e < a.off[u + 1]; e += blockDim.x) {
        const int s = a.idx[e];
        const double q2 = a.s_mom[2 * s + 1];
#pragma unroll
        for (int k = 0; k < NS; k++) {
            const double dx = px[k] - a.s_ctr[3 * s], dy = py[k] - a.s_ctr[3 * s + 1], dz = pz[k] - a.s_ctr[3 * s + 2];
            phi2 += q2 * q2 / (dx * dx + dy * dy + dz * dz);
        }
    }
    // near field: a leaf farther than twice its radius from a sampled
    // target adds |q_L|_2^2 / d^2, as a cluster entry does; a closer one
    // adds each particle's q^2 / r^2 with r no smaller than the leaf's mean
    // particle spacing (radius / count^(1/3)), which keeps a chance close
    // neighbour from dominating the estimate; FP32 (an estimate)
    float near = 0.0f;
    for (int64_t e = d_off[u]; e < d_off[u + 1]; e++) {
        const int s = d_idx[e], b = s_ibeg[s], m = a.s_numpar[s];
        const double rs = a.s_rad[s], q2 = a.s_mom[2 * s + 1];
        bool touch[NS], any = false;
#pragma unroll
        for (int k = 0; k < NS; k++) {
            const double dx = px[k] - a.s_ctr[3 * s], dy = py[k] - a.s_ctr[3 * s + 1], dz = pz[k] - a.s_ctr[3 * s + 2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            touch[k] = d2 <= 4.0 * rs * rs;
            any = any || touch[k];
            if (!touch[k] && threadIdx.x == 0) phi2 += q2 * q2 / d2;
        }
        if (!any) continue;
        const float h = (float)(rs / cbrt((double)m));
        const float h2 = fmaxf(h * h, FLT_MIN);
        for (int j = threadIdx.x; j < m; j += blockDim.x) {
            const float q = (float)sq[b + j];
#pragma unroll
            for (int k = 0; k < NS; k++) {
                if (!touch[k]) continue;
                const float dx = (float)(px[k] - sx[b + j]), dy = (float)(py[k] - sy[b + j]),
                            dz = (float)(pz[k] - sz[b + j]);
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                if (r2 > 0.0f) near += q * q / fmaxf(r2, h2);
            }
        }
    }
    phi2 += (double)near;
    __shared__ double red[128];
    red[threadIdx.x] = phi2;
    __syncthreads();
    for (int h = 64; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        unit_sums[2 * u] = nt * red[0] / NS;
        unit_sums[2 * u + 1] = (double)nt * (double)(a.off[u + 1] - a.off[u]);
    }
}

// One block per system: its share from the sums over its units (leaves
// sys_off[k] .. sys_off[k+1]), added in a fixed order (deterministic).
__global__ void k_system_share(const int *__restrict__ sys_off, const double *__restrict__ unit_sums, double c_tol,
                               float *__restrict__ log_share)
{
    __shared__ double sp[256], sn[256];
    const int k = blockIdx.x;
    double p = 0.0, n = 0.0;
    for (int u = sys_off[k] + threadIdx.x; u < sys_off[k + 1]; u += blockDim.x) {
        p += unit_sums[2 * u];
        n += unit_sums[2 * u + 1];
    }
    sp[threadIdx.x] = p;
    sn[threadIdx.x] = n;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) { sp[threadIdx.x] += sp[threadIdx.x + s]; sn[threadIdx.x] += sn[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double share = sn[0] > 0.0 ? c_tol * sqrt(sp[0] / sn[0]) : 0.0;
        log_share[k] = share > 0.0 ? (float)log10(share) : -1.0e30f;
    }
}

__global__ void k_select_share(FeatureArgs a, int nsys, const int *__restrict__ sys_off, int64_t n,
                               const float *__restrict__ pred, const float *__restrict__ feat,
                               const float *__restrict__ log_share, unsigned char *__restrict__ choice)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n) return;
    int lo = 0, hi = a.units;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (a.off[mid] <= e) lo = mid; else hi = mid;
    }
    int k0 = 0, k1 = nsys;                 // the unit's system
    while (k1 - k0 > 1) {
        const int mid = (k0 + k1) >> 1;
        if (sys_off[mid] <= lo) k0 = mid; else k1 = mid;
    }
    const int tn = a.unit_node[lo], s = a.idx[e];
    const double dx = a.t_ctr[3 * tn] - a.s_ctr[3 * s], dy = a.t_ctr[3 * tn + 1] - a.s_ctr[3 * s + 1],
                 dz = a.t_ctr[3 * tn + 2] - a.s_ctr[3 * s + 2];
    const double scale = a.s_mom[2 * s + 1] / sqrt(dx * dx + dy * dy + dz * dz);
    const float budget = scale > 0.0 ? log_share[k0] - (float)log10(scale) : 1.0e30f;
    unsigned char c = MLP_PP;
    for (int d = MLP_DMIN; d <= MLP_DMAX; d++) {
        if (pred[e * MLP_OUT + (d - MLP_DMIN)] <= budget) { c = (unsigned char)d; break; }
    }
    const float ns = exp10f(feat[e * MLP_IN + 0]);
    if (c != MLP_PP) {
        const float P = (float)((c + 1) * (c + 1) * (c + 1));
        if (P >= ns) c = MLP_PP;
    }
    choice[e] = c;
}

void launch_select_share(const FeatureArgs &a, int nsys, const int *sys_off, const int *t_ibeg, const int64_t *d_off,
                         const int *d_idx, const int *s_ibeg, const double *sx, const double *sy, const double *sz,
                         const double *sq, const double *tx, const double *ty, const double *tz, double c_tol,
                         int64_t n, const float *pred, const float *feat, double *unit_sums, float *log_share,
                         unsigned char *choice, cudaStream_t st)
{
    if (n <= 0 || a.units <= 0 || nsys <= 0) return;
    k_unit_phi2_sampled<<<a.units, 128, 0, st>>>(a, t_ibeg, d_off, d_idx, s_ibeg, sx, sy, sz, sq, tx, ty, tz,
                                                  unit_sums);
    k_system_share<<<nsys, 256, 0, st>>>(sys_off, unit_sums, c_tol, log_share);
    k_select_share<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, nsys, sys_off, n, pred, feat, log_share, choice);
}


}  // namespace bt
