// bt_sym.cu -- symmetric near-field pairs of the mixed path.
//
// When the targets are the sources (same particles, same tree) and the
// kernel is symmetric in r (Coulomb, Yukawa, regularized Coulomb), a pair of
// distinct leaves {A, B} that each hold the other in their near-field list
// needs each pair distance once: 1/r_ij serves both phi_i (i in A, source j
// in B) and phi_j (j in B, source i in A).  The reference evaluates the two
// directions separately (src/interaction_compute/interaction_compute_pc.c,
// direct list of each target batch); the sums are the same up to rounding.
// Pairs of leaves whose boxes lie within the close-pair distance of each
// other (touching leaves, mostly) can hold close pairs, which the mixed path
// evaluates in FP64 from the FP64 particles.  Their kernel (CLAMP) raises
// every FP32 r^2 to at least the close-pair distance squared, so a close
// pair adds a bounded, known term (the kernel at that distance) to both
// sides; before the main loop the block finds the particles of each leaf
// that lie within that distance of the other leaf's box (a few per cent of
// them, found in FP64), recomputes the FP32 r^2 of every pair among those
// candidates with the main loop's own instructions, and for each pair
// below the distance writes the FP64 kernel minus the clamped term into
// both sides' slices.  The main loop's sums are added to these at the end.
// Self pairs (A with A) stay in the particle-output kernel.
//
// Work: one block per pair.  The block's threads hold A's targets, four per
// thread in two packed FP32 pairs, in chunks of 512; B's particles stream
// through shared memory, staged as {v, v} pairs.  Every 1/r feeds the
// thread's A-side sums and, through a per-thread register per source, the
// B side: each group of 16 sources is reduced across the warp by a
// reduce-scatter (16 shuffles for 16 sources; lanes 2i and 2i+1 end with
// source i), then across the block's warps in a fixed order.  Both sides go to the
// pair's own slices of a partial-sum array; k_sym_gather adds each leaf's
// slices in FP64 in pair order.  No atomics: the potentials are the same bit
// for bit on every run.
#include <cuda_runtime.h>

#include <cstdint>

#include <cfloat>

#include "bt_f2.cuh"
#include "bt_kernels.cuh"
#include "bt_mixed.h"
#include "bt_sym.h"

namespace bt {

namespace {

constexpr int SY_THREADS = 128;
// targets of A per thread (packed in pairs) and the resident blocks per SM
// the register budget is sized for; build-time choices.  Measured on the 16M
// clustered step: 4 and 6 (856 ms) against 6 and 4 (872 ms), 8 and 4
// (886 ms), 8 and 3 (894 ms)
#ifndef BT_SYM_TPT
#define BT_SYM_TPT 4
#endif
#ifndef BT_SYM_MIN_BLOCKS
#define BT_SYM_MIN_BLOCKS 6
#endif
constexpr int SY_TPT = BT_SYM_TPT;
constexpr int SY_NP = SY_TPT / 2;
constexpr int SY_CHUNK = SY_TPT * SY_THREADS;  // targets of A per pass
constexpr int SY_TILE = 512;                   // sources of B per shared-memory tile
constexpr int SY_SB = 16;                      // sources per warp reduction
constexpr int SY_WARPS = SY_THREADS / 32;
constexpr float SY_PAD_POS = 1.0e18f;          // padding sources: far away, no charge

// v[0..2H-1] per lane -> v[0..H-1]: lanes with bit LX of their index keep
// the upper half of the indices, the others the lower half, each adding the
// partner's (lane ^ LX) copy of the half it keeps.
template <int H, int LX>
__device__ __forceinline__ void rs_stage(float *v, int lane)
{
    const bool up = (lane & LX) != 0;
#pragma unroll
    for (int i = 0; i < H; i++) {
        const float a = v[i], b = v[i + H];
        const float keep = up ? b : a, send = up ? a : b;
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, LX);
    }
}

// The kernel value of a packed pair of r^2 (the particle-output kernel's
// arithmetic): Coulomb 1/r; regularised Coulomb 1/sqrt(r^2 + eps^2);
// Yukawa with one Newton step on 1/r, then exp(-kappa r) by ex2.
template <int KT>
__device__ __forceinline__ f2_t sym_kval(f2_t r2, f2_t kc2)
{
    if (KT == 3) r2 = f2_fma(f2_make(1.0f, 1.0f), kc2, r2);
    float ra, rb;
    f2_split(r2, ra, rb);
    f2_t k = f2_make(rsqrt_apx(ra), rsqrt_apx(rb));
    if (KT == 2) {
        const f2_t h = f2_mul(r2, k);
        const f2_t t = f2_fma(f2_mul(h, f2_make(-0.5f, -0.5f)), k, f2_make(1.5f, 1.5f));
        float e0, e1;
        f2_split(f2_mul(kc2, f2_mul(h, t)), e0, e1);
        k = f2_mul(f2_mul(k, t), f2_make(ex2_apx(e0), ex2_apx(e1)));
    }
    return k;
}

// The main loop's FP32 r^2 of one pair, with its instructions: x, y, z the
// target in the source leaf's frame, p the source.
__device__ __forceinline__ float sym_r2(float x, float y, float z, float4 p)
{
    const f2_t dx = f2_sub(f2_make(x, x), f2_make(p.x, p.x)), dy = f2_sub(f2_make(y, y), f2_make(p.y, p.y)),
               dz = f2_sub(f2_make(z, z), f2_make(p.z, p.z));
    float r2, unused;
    f2_split(f2_fma(dx, dx, f2_fma(dy, dy, f2_mul(dz, dz))), r2, unused);
    return r2;
}

// Indices i < n of the particles (FP64, from `base`) within distance d of
// the box b (x0 x1 y0 y1 z0 z1), in index order, into out; returns how many.
__device__ int near_box(int *out, int n, int base, const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, const double *b, double d, int *wcnt)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int total = 0;
    for (int c0 = 0; c0 < n; c0 += SY_THREADS) {
        const int i = c0 + threadIdx.x;
        bool f = false;
        if (i < n) {
            const double px = x[base + i], py = y[base + i], pz = z[base + i];
            const double gx = fmax(0.0, fmax(b[0] - px, px - b[1])), gy = fmax(0.0, fmax(b[2] - py, py - b[3])),
                         gz = fmax(0.0, fmax(b[4] - pz, pz - b[5]));
            f = gx * gx + gy * gy + gz * gz <= d * d;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, f);
        if (lane == 0) wcnt[warp] = __popc(bal);
        __syncthreads();
        int off = total, all = 0;
#pragma unroll
        for (int w = 0; w < SY_WARPS; w++) {
            off += w < warp ? wcnt[w] : 0;
            all += wcnt[w];
        }
        if (f) out[off + __popc(bal & ((1u << lane) - 1u))] = i;
        __syncthreads();
        total += all;
    }
    return total;
}

template <int KT, bool CLAMP>
__global__ void __launch_bounds__(SY_THREADS, BT_SYM_MIN_BLOCKS) k_pp_sym(SymArgs a)
{
    __shared__ __align__(16) f2_t tile[SY_TILE][4];     // {x, x}, {y, y}, {z, z}, {q, q}
    __shared__ float red[SY_WARPS][SY_TILE];
    __shared__ float accB[SYM_MAX_LEAF];
    __shared__ double accA[SY_TPT][SY_THREADS];          // A side: each tile's FP32 sums, added in FP64
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int2 pr = a.pair[blockIdx.x];
    const int A = pr.x, B = pr.y;
    const int ia = a.ibeg[A], na = a.numpar[A], ib = a.ibeg[B], nb = a.numpar[B];
    float *outA = a.partial + a.slot[blockIdx.x];
    float *outB = outA + na;
    // A's targets in B's frame: positions relative to A's centre minus the offset of B's
    const float ox = (float)(a.ctr[3 * B] - a.ctr[3 * A]), oy = (float)(a.ctr[3 * B + 1] - a.ctr[3 * A + 1]),
                oz = (float)(a.ctr[3 * B + 2] - a.ctr[3 * A + 2]);
    const f2_t kc2 = f2_make(a.kc, a.kc);
    // the close-pair distance squared, as the particle-output kernel has it
    float thr2 = 0.0f;
    if (CLAMP) {
        const double rr = MX_CLOSE_FRAC * (a.rad[A] + a.rad[B]);
        thr2 = fmaxf((float)(rr * rr), FLT_MIN);
        __shared__ int wcnt[SY_WARPS];
        int *candA = reinterpret_cast<int *>(&tile[0][0]), *candB = candA + SYM_MAX_LEAF;
        for (int i = threadIdx.x; i < na; i += SY_THREADS) outA[i] = 0.0f;
        for (int j = threadIdx.x; j < nb; j += SY_THREADS) outB[j] = 0.0f;
        // every pair with FP32 r^2 below thr2 lies within 1.01 thr of both boxes
        const double d = 1.01 * sqrt((double)thr2);
        const int nca = near_box(candA, na, ia, a.x64, a.y64, a.z64, a.box + 6 * B, d, wcnt);
        const int ncb = near_box(candB, nb, ib, a.x64, a.y64, a.z64, a.box + 6 * A, d, wcnt);
        if (nca > 0 && ncb > 0) {
            float kcl, unused;
            f2_split(sym_kval<KT>(f2_make(thr2, thr2), kc2), kcl, unused);   // the clamped term's kernel value
            const double kcd = (double)kcl;
            for (int k = threadIdx.x; k < nca + ncb; k += SY_THREADS) {
                // thread k: candidate k of A (its sum over B's candidates), then of B
                const bool sideA = k < nca;
                const int i = sideA ? candA[k] : candB[k - nca];
                const int gi = (sideA ? ia : ib) + i;
                const float4 pi = a.pos[gi];
                double c = 0.0;
                for (int m = 0; m < (sideA ? ncb : nca); m++) {
                    const int j = sideA ? candB[m] : candA[m];
                    const int gj = (sideA ? ib : ia) + j;
                    const float4 pj = a.pos[gj];
                    // the pair's r^2 as the main loop forms it: A's target in B's frame
                    const float r2 = sideA ? sym_r2(pi.x - ox, pi.y - oy, pi.z - oz, pj)
                                           : sym_r2(pj.x - ox, pj.y - oy, pj.z - oz, pi);
                    if (r2 < thr2) {
                        const double ex = a.x64[gi] - a.x64[gj], ey = a.y64[gi] - a.y64[gj],
                                     ez = a.z64[gi] - a.z64[gj];
                        c += k_pp<KT>(ex * ex + ey * ey + ez * ez, a.q64[gj], a.kp) - (double)pj.w * kcd;
                    }
                }
                (sideA ? outA[i] : outB[i]) = (float)c;
            }
        }
        __syncthreads();                                  // the candidate lists live in the tile
    }
    for (int j = threadIdx.x; j < nb; j += SY_THREADS) accB[j] = 0.0f;
    for (int c0 = 0; c0 < na; c0 += SY_CHUNK) {
        // targets c0 + threadIdx.x + k * SY_THREADS, k = 0..SY_TPT-1, packed as (0, 1), (2, 3), ...
        f2_t X[SY_NP], Y[SY_NP], Z[SY_NP], QT[SY_NP], S[SY_NP];
        bool act[SY_TPT];
#pragma unroll
        for (int p = 0; p < SY_NP; p++) {
            const int t0 = c0 + threadIdx.x + (2 * p) * SY_THREADS, t1 = t0 + SY_THREADS;
            act[2 * p] = t0 < na;
            act[2 * p + 1] = t1 < na;
            const float4 p0 = a.pos[ia + (act[2 * p] ? t0 : 0)], p1 = a.pos[ia + (act[2 * p + 1] ? t1 : 0)];
            X[p] = f2_make(p0.x - ox, p1.x - ox);
            Y[p] = f2_make(p0.y - oy, p1.y - oy);
            Z[p] = f2_make(p0.z - oz, p1.z - oz);
            QT[p] = f2_make(act[2 * p] ? p0.w : 0.0f, act[2 * p + 1] ? p1.w : 0.0f);   // absent targets add nothing
            S[p] = f2_make(0.0f, 0.0f);
        }
#pragma unroll
        for (int k = 0; k < SY_TPT; k++) accA[k][threadIdx.x] = 0.0;
        for (int s0 = 0; s0 < nb; s0 += SY_TILE) {
            const int cm = min(SY_TILE, nb - s0), cmb = (cm + SY_SB - 1) & ~(SY_SB - 1);
            __syncthreads();                              // the previous tile is done with
            for (int i = threadIdx.x; i < cmb; i += SY_THREADS) {
                const float4 p = i < cm ? a.pos[ib + s0 + i] : make_float4(SY_PAD_POS, SY_PAD_POS, SY_PAD_POS, 0.0f);
                tile[i][0] = f2_make(p.x, p.x);
                tile[i][1] = f2_make(p.y, p.y);
                tile[i][2] = f2_make(p.z, p.z);
                tile[i][3] = f2_make(p.w, p.w);
            }
            __syncthreads();
            for (int sb = 0; sb < cmb; sb += SY_SB) {
                float v[SY_SB];
#pragma unroll
                for (int s = 0; s < SY_SB; s++) {
                    const ulonglong2 xy = *reinterpret_cast<const ulonglong2 *>(&tile[sb + s][0]);
                    const ulonglong2 zq = *reinterpret_cast<const ulonglong2 *>(&tile[sb + s][2]);
                    f2_t cb = f2_make(0.0f, 0.0f);
#pragma unroll
                    for (int p = 0; p < SY_NP; p++) {
                        const f2_t dx = f2_sub(X[p], xy.x), dy = f2_sub(Y[p], xy.y), dz = f2_sub(Z[p], zq.x);
                        f2_t r2 = f2_fma(dx, dx, f2_fma(dy, dy, f2_mul(dz, dz)));
                        if (CLAMP) {
                            float ra, rb;
                            f2_split(r2, ra, rb);
                            r2 = f2_make(fmaxf(ra, thr2), fmaxf(rb, thr2));
                        }
                        const f2_t rinv = sym_kval<KT>(r2, kc2);      // serves both sides
                        S[p] = f2_fma(zq.y, rinv, S[p]);
                        // B side: the targets' charges over r, folded into one pair
                        cb = p == 0 ? f2_mul(QT[0], rinv) : f2_fma(QT[p], rinv, cb);
                    }
                    float c0v, c1v;
                    f2_split(cb, c0v, c1v);
                    v[s] = c0v + c1v;
                }
                // reduce-scatter over the warp: lanes 2i and 2i+1 end with source i
                rs_stage<8, 16>(v, lane);
                rs_stage<4, 8>(v, lane);
                rs_stage<2, 4>(v, lane);
                rs_stage<1, 2>(v, lane);
                v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
                if ((lane & 1) == 0) red[warp][sb + (lane >> 1)] = v[0];
            }
            // the tile's A-side sums into FP64 (FP32 chains of at most one tile)
#pragma unroll
            for (int p = 0; p < SY_NP; p++) {
                float lo, hi;
                f2_split(S[p], lo, hi);
                accA[2 * p][threadIdx.x] += (double)lo;
                accA[2 * p + 1][threadIdx.x] += (double)hi;
                S[p] = f2_make(0.0f, 0.0f);
            }
            __syncthreads();
            // the block's B-side sum per source, warps in a fixed order
            for (int j = threadIdx.x; j < cm; j += SY_THREADS) {
                float r = red[0][j];
#pragma unroll
                for (int w = 1; w < SY_WARPS; w++) r += red[w][j];
                accB[s0 + j] += r;
            }
        }
#pragma unroll
        for (int k = 0; k < SY_TPT; k++) {
            const int t = c0 + threadIdx.x + k * SY_THREADS;
            if (act[k]) outA[t] = (float)(CLAMP ? accA[k][threadIdx.x] + (double)outA[t] : accA[k][threadIdx.x]);
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < nb; j += SY_THREADS) outB[j] = CLAMP ? accB[j] + outB[j] : accB[j];
}

__global__ void k_sym_gather(SymGatherArgs a)
{
    const int u = blockIdx.x;
    const int64_t k0 = a.in_off[u], k1 = a.in_off[u + 1];
    if (k0 == k1) return;
    const int node = a.leaf_node[u];
    const int ib = a.ibeg[node], nb = a.numpar[node];
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        double s = 0.0;
        for (int64_t k = k0; k < k1; k++) s += (double)a.partial[a.in_slot[k] + j];
        a.pot[ib + j] += s;
    }
}

}  // namespace

void launch_pp_sym(int kernel, const SymArgs &a, cudaStream_t st)
{
    if (a.npairs <= 0) return;
    if (kernel == 3) k_pp_sym<3, false><<<a.npairs, SY_THREADS, 0, st>>>(a);
    else if (kernel == 2) k_pp_sym<2, false><<<a.npairs, SY_THREADS, 0, st>>>(a);
    else k_pp_sym<1, false><<<a.npairs, SY_THREADS, 0, st>>>(a);
}

void launch_pp_sym_close(int kernel, const SymArgs &a, cudaStream_t st)
{
    if (a.npairs <= 0) return;
    if (kernel == 3) k_pp_sym<3, true><<<a.npairs, SY_THREADS, 0, st>>>(a);
    else if (kernel == 2) k_pp_sym<2, true><<<a.npairs, SY_THREADS, 0, st>>>(a);
    else k_pp_sym<1, true><<<a.npairs, SY_THREADS, 0, st>>>(a);
}

void launch_sym_gather(const SymGatherArgs &a, cudaStream_t st)
{
    if (a.nleaves > 0) k_sym_gather<<<a.nleaves, 128, 0, st>>>(a);
}

}  // namespace bt
