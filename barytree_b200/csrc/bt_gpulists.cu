// bt_gpulists.cu -- particle-cluster / cluster-particle interaction lists
// traversed on the GPU.
//
// pc_compute_interaction_list (src/interaction_lists/interaction_lists.c:464-533)
// walks the source tree depth first for one target batch: a node whose
// radius plus the batch's radius is below theta times the centre distance,
// whose radius is not zero and which holds more particles than size check
// times the grid size becomes a cluster (approximation) entry; otherwise a
// leaf becomes a direct entry and an internal node is opened, children in
// order.  Here one thread walks one batch with an explicit stack in shared
// memory (interleaved by thread, so lanes at the same depth hit different
// banks); popping the top and pushing the children last-first visits nodes
// in the recursion's order.  The comparisons use __dsub_rn / __dmul_rn /
// __dadd_rn / __dsqrt_rn, so nothing is contracted into an FMA and every
// value equals the host's IEEE FP64 result: membership and order are the
// host traversal's (and the reference's) bit for bit.
//
// Two passes: count the entries of every batch, prefix sums on the host,
// then write them.  The node geometry of the traversed tree is small
// (tens of thousands of nodes) and stays in L1/L2 across the threads.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bt_gpulists.h"

namespace bt {

namespace {

constexpr int GL_THREADS = 64;
constexpr int GL_MAX_STACK = 384;          // shared-memory stack slots per thread (98 KB per block)

template <bool FILL>
__global__ void __launch_bounds__(GL_THREADS)
k_pc_traverse(int nb, const double4 *__restrict__ bat, const int *__restrict__ broot,
              const double4 *__restrict__ geo, const int2 *__restrict__ cnt_nc, const int *__restrict__ child,
              double theta, double thr, int depth_cap, int *__restrict__ counts, const int64_t *__restrict__ aoff,
              const int64_t *__restrict__ poff, int *__restrict__ aidx, int *__restrict__ pidx,
              int *__restrict__ overflow)
{
    extern __shared__ int stk[];
    const int b = blockIdx.x * GL_THREADS + threadIdx.x;
    if (b >= nb) return;
    const double4 B = bat[b];
    int sp = 0, na = 0, np = 0;
    int *a_out = FILL ? aidx + aoff[b] : nullptr, *p_out = FILL ? pidx + poff[b] : nullptr;
    const int root = broot[b];
    if (root >= 0) stk[threadIdx.x] = root, sp = 1;
    while (sp) {
        sp--;
        const int node = stk[sp * GL_THREADS + threadIdx.x];
        const double4 g = geo[node];
        const double tx = __dsub_rn(B.x, g.x), ty = __dsub_rn(B.y, g.y), tz = __dsub_rn(B.z, g.z);
        const double dist = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(tx, tx), __dmul_rn(ty, ty)), __dmul_rn(tz, tz)));
        const int2 cn = cnt_nc[node];      // numpar, nchild
        if (__dadd_rn(g.w, B.w) < __dmul_rn(dist, theta) && g.w != 0.0 && thr < (double)cn.x) {
            if (FILL) a_out[na] = node;
            na++;
        } else if (cn.y == 0) {
            if (FILL) p_out[np] = node;
            np++;
        } else {
            if (sp + cn.y > depth_cap) {
                atomicExch(overflow, 1);
                return;
            }
            for (int i = cn.y - 1; i >= 0; i--) stk[(sp++) * GL_THREADS + threadIdx.x] = child[8 * (size_t)node + i];
        }
    }
    if (!FILL) {
        counts[b] = na;
        counts[nb + b] = np;
    }
}

}  // namespace

int gpu_pc_lists(const bt_tree *trav, const bt_tree *bat, const bt_params *o, void *work, size_t work_bytes,
                 bt_csr *ap, bt_csr *pp, cudaStream_t st, long long *launches)
{
    const int nb = bat->nleaves, nn = trav->n;
    if (nb <= 0 || nn <= 0) return -1;
    const int cap = 7 * trav->max_depth + 8;
    if (cap > GL_MAX_STACK) return -1;
    // device layout: geometry, counts/children, batches, roots, counts,
    // overflow flag, then offsets and entries
    char *p = (char *)work, *end = p + work_bytes;
    auto take = [&](size_t bytes) -> void * {
        char *r = p;
        p += (bytes + 255) & ~size_t(255);
        return p <= end ? r : nullptr;
    };
    double4 *d_geo = (double4 *)take(sizeof(double4) * (size_t)nn);
    int2 *d_cn = (int2 *)take(sizeof(int2) * (size_t)nn);
    int *d_child = (int *)take(sizeof(int) * 8 * (size_t)nn);
    double4 *d_bat = (double4 *)take(sizeof(double4) * (size_t)nb);
    int *d_root = (int *)take(sizeof(int) * (size_t)nb);
    int *d_cnt = (int *)take(sizeof(int) * 2 * (size_t)nb);
    int *d_ovf = (int *)take(sizeof(int));
    int64_t *d_off = (int64_t *)take(sizeof(int64_t) * 2 * ((size_t)nb + 1));
    if (!d_off) return -1;

    std::vector<double4> geo(nn), bg(nb);
    std::vector<int2> cn(nn);
    std::vector<int> root(nb);
    for (int i = 0; i < nn; i++) {
        geo[i] = make_double4(trav->xm[i], trav->ym[i], trav->zm[i], trav->rad[i]);
        cn[i] = make_int2(trav->numpar[i], trav->nchild[i]);
    }
    for (int i = 0; i < nb; i++) {
        const int leaf = bat->leaves[i];
        bg[i] = make_double4(bat->xm[leaf], bat->ym[leaf], bat->zm[leaf], bat->rad[leaf]);
    }
    // the batch's system: the traversed tree's root of the same system
    for (int k = 0; k < bat->nroots; k++)
        for (int i = bat->leaf_off[k]; i < bat->leaf_off[k + 1]; i++) root[i] = trav->roots[k];

    cudaError_t e;
#define GL_CK(x) do { if ((e = (x)) != cudaSuccess) return (int)e; } while (0)
    GL_CK(cudaMemcpyAsync(d_geo, geo.data(), sizeof(double4) * (size_t)nn, cudaMemcpyHostToDevice, st));
    GL_CK(cudaMemcpyAsync(d_cn, cn.data(), sizeof(int2) * (size_t)nn, cudaMemcpyHostToDevice, st));
    GL_CK(cudaMemcpyAsync(d_child, trav->child, sizeof(int) * 8 * (size_t)nn, cudaMemcpyHostToDevice, st));
    GL_CK(cudaMemcpyAsync(d_bat, bg.data(), sizeof(double4) * (size_t)nb, cudaMemcpyHostToDevice, st));
    GL_CK(cudaMemcpyAsync(d_root, root.data(), sizeof(int) * (size_t)nb, cudaMemcpyHostToDevice, st));
    GL_CK(cudaMemsetAsync(d_ovf, 0, sizeof(int), st));
    const size_t smem = sizeof(int) * (size_t)GL_THREADS * (size_t)cap;
    GL_CK(cudaFuncSetAttribute(k_pc_traverse<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    GL_CK(cudaFuncSetAttribute(k_pc_traverse<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const double thr = o->size_check * o->P;
    const int blocks = (nb + GL_THREADS - 1) / GL_THREADS;
    k_pc_traverse<false><<<blocks, GL_THREADS, smem, st>>>(nb, d_bat, d_root, d_geo, d_cn, d_child, o->theta, thr,
                                                           cap, d_cnt, nullptr, nullptr, nullptr, nullptr, d_ovf);
    GL_CK(cudaGetLastError());
    std::vector<int> cnt(2 * (size_t)nb + 1);
    GL_CK(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * 2 * (size_t)nb, cudaMemcpyDeviceToHost, st));
    GL_CK(cudaMemcpyAsync(cnt.data() + 2 * (size_t)nb, d_ovf, sizeof(int), cudaMemcpyDeviceToHost, st));
    GL_CK(cudaStreamSynchronize(st));
    *launches += 1;
    if (cnt[2 * (size_t)nb]) return -1;

    std::vector<int64_t> off(2 * ((size_t)nb + 1));
    int64_t *aoff = off.data(), *poff = aoff + nb + 1;
    aoff[0] = poff[0] = 0;
    for (int i = 0; i < nb; i++) {
        aoff[i + 1] = aoff[i] + cnt[i];
        poff[i + 1] = poff[i] + cnt[nb + i];
    }
    const int64_t na = aoff[nb], np = poff[nb];
    int *d_aidx = (int *)take(sizeof(int) * (size_t)(na > 0 ? na : 1));
    int *d_pidx = (int *)take(sizeof(int) * (size_t)(np > 0 ? np : 1));
    if (!d_aidx || !d_pidx) return -1;
    GL_CK(cudaMemcpyAsync(d_off, off.data(), sizeof(int64_t) * off.size(), cudaMemcpyHostToDevice, st));
    k_pc_traverse<true><<<blocks, GL_THREADS, smem, st>>>(nb, d_bat, d_root, d_geo, d_cn, d_child, o->theta, thr,
                                                          cap, nullptr, d_off, d_off + nb + 1, d_aidx, d_pidx, d_ovf);
    GL_CK(cudaGetLastError());
    *launches += 1;
    bt_csr *out[2] = {ap, pp};
    int *didx[2] = {d_aidx, d_pidx};
    const int64_t *hoff[2] = {aoff, poff};
    for (int k = 0; k < 2; k++) {
        bt_csr *c = out[k];
        c->rows = nb;
        c->off = (int64_t *)malloc(sizeof(int64_t) * ((size_t)nb + 1));
        memcpy(c->off, hoff[k], sizeof(int64_t) * ((size_t)nb + 1));
        const int64_t m = hoff[k][nb];
        c->idx = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
        if (m) GL_CK(cudaMemcpyAsync(c->idx, didx[k], sizeof(int) * (size_t)m, cudaMemcpyDeviceToHost, st));
    }
    GL_CK(cudaStreamSynchronize(st));
#undef GL_CK
    return 0;
}

}  // namespace bt
