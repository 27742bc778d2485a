// bt_sym.cu -- symmetric near-field pairs of the mixed path.
//
// When the targets are the sources (same particles, same tree) and the
// kernel is symmetric in r (Coulomb, regularized Coulomb), a pair of
// distinct leaves {A, B} that each hold the other in their near-field list
// needs each pair distance once: 1/r_ij serves both phi_i (i in A, source j
// in B) and phi_j (j in B, source i in A).  The reference evaluates the two
// directions separately (src/interaction_compute/interaction_compute_pc.c,
// direct list of each target batch); the sums are the same up to rounding.
// Only pairs whose leaf boxes are too far apart to hold a close pair (the
// mixed path's FP64 rule) are taken here; the rest stay in the
// particle-output kernel.
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

#include "bt_f2.cuh"
#include "bt_sym.h"

namespace bt {

namespace {

constexpr int SY_THREADS = 128;
constexpr int SY_TPT = 4;                      // targets of A per thread: two packed pairs
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

template <int KT>
__global__ void __launch_bounds__(SY_THREADS, 6) k_pp_sym(SymArgs a)
{
    __shared__ __align__(16) f2_t tile[SY_TILE][4];     // {x, x}, {y, y}, {z, z}, {q, q}
    __shared__ float red[SY_WARPS][SY_TILE];
    __shared__ float accB[SYM_MAX_LEAF];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int2 pr = a.pair[blockIdx.x];
    const int A = pr.x, B = pr.y;
    const int ia = a.ibeg[A], na = a.numpar[A], ib = a.ibeg[B], nb = a.numpar[B];
    float *outA = a.partial + a.slot[blockIdx.x];
    float *outB = outA + na;
    // A's targets in B's frame: positions relative to A's centre minus the offset of B's
    const float ox = (float)(a.ctr[3 * B] - a.ctr[3 * A]), oy = (float)(a.ctr[3 * B + 1] - a.ctr[3 * A + 1]),
                oz = (float)(a.ctr[3 * B + 2] - a.ctr[3 * A + 2]);
    const f2_t kc2 = f2_make(a.kc, a.kc), one = f2_make(1.0f, 1.0f);
    for (int j = threadIdx.x; j < nb; j += SY_THREADS) accB[j] = 0.0f;
    for (int c0 = 0; c0 < na; c0 += SY_CHUNK) {
        // targets c0 + threadIdx.x + k * SY_THREADS, k = 0..3, packed as (0, 1), (2, 3)
        f2_t X[2], Y[2], Z[2], QT[2], S[2];
        bool act[SY_TPT];
#pragma unroll
        for (int p = 0; p < 2; p++) {
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
                    f2_t rinv[2];
#pragma unroll
                    for (int p = 0; p < 2; p++) {
                        const f2_t dx = f2_sub(X[p], xy.x), dy = f2_sub(Y[p], xy.y), dz = f2_sub(Z[p], zq.x);
                        f2_t r2 = f2_fma(dx, dx, f2_fma(dy, dy, f2_mul(dz, dz)));
                        if (KT == 3) r2 = f2_fma(one, kc2, r2);
                        float ra, rb;
                        f2_split(r2, ra, rb);
                        rinv[p] = f2_make(rsqrt_apx(ra), rsqrt_apx(rb));
                        S[p] = f2_fma(zq.y, rinv[p], S[p]);
                    }
                    // B side: the four targets' charges over r, folded into one value
                    float c0v, c1v;
                    f2_split(f2_fma(QT[0], rinv[0], f2_mul(QT[1], rinv[1])), c0v, c1v);
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
        for (int p = 0; p < 2; p++) {
            float lo, hi;
            f2_split(S[p], lo, hi);
            const int t0 = c0 + threadIdx.x + (2 * p) * SY_THREADS, t1 = t0 + SY_THREADS;
            if (act[2 * p]) outA[t0] = lo;
            if (act[2 * p + 1]) outA[t1] = hi;
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < nb; j += SY_THREADS) outB[j] = accB[j];
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
    if (kernel == 3) k_pp_sym<3><<<a.npairs, SY_THREADS, 0, st>>>(a);
    else k_pp_sym<1><<<a.npairs, SY_THREADS, 0, st>>>(a);
}

void launch_sym_gather(const SymGatherArgs &a, cudaStream_t st)
{
    if (a.nleaves > 0) k_sym_gather<<<a.nleaves, 128, 0, st>>>(a);
}

}  // namespace bt
