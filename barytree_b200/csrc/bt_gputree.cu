// bt_gputree.cu -- the adaptive tree built on the GPU, level by level.
//
// Same node sets, boxes, radii, numbering and particle ranges as the host
// build (bt_tree.c) and the reference (src/tree/tree_linked_list.c:16-293,
// src/tree/partition.c:14-392): per level,
//   1. bounding boxes of the level's nodes: exact min/max through atomics on
//      order-preserving 64-bit keys of the FP64 coordinates;
//   2. the host applies the reference's split rule to the boxes (the same
//      FP64 arithmetic as bt_tree.c);
//   3. per divided axis, in the reference's order x, y, z, every particle's
//      child slot bit: a part of two or more particles sends {a <= mid} low,
//      a part of exactly one sends it low only if a < mid (partition.c:75-79);
//   4. a stable scatter into the child ranges (first divided axis most
//      significant in memory, as the reference's successive binary splits).
// Particles never leave the GPU; the host receives only per-node boxes and
// slot counts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bt_gputree.h"

namespace bt {

namespace {

constexpr int GT_CHUNK = 4096;
constexpr int GT_THREADS = 256;

__device__ __forceinline__ unsigned long long dkey(double v)
{
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}

__host__ __device__ inline double dkey_inv(unsigned long long k)
{
    unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
    double v;
    memcpy(&v, &b, sizeof v);
    return v;
}

struct ChunkArgs {
    const int *chunk_node;      // chunk -> level-local node
    const int *chunk_begin;     // chunk -> first particle (absolute)
    const int *chunk_len;
};

__global__ void k_boxes(ChunkArgs c, const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, unsigned long long *__restrict__ kmin,
                        unsigned long long *__restrict__ kmax)
{
    const int ch = blockIdx.x, node = c.chunk_node[ch], b = c.chunk_begin[ch], n = c.chunk_len[ch];
    unsigned long long mn[3] = {~0ULL, ~0ULL, ~0ULL}, mx[3] = {0, 0, 0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        unsigned long long k0 = dkey(x[b + i]), k1 = dkey(y[b + i]), k2 = dkey(z[b + i]);
        mn[0] = min(mn[0], k0); mx[0] = max(mx[0], k0);
        mn[1] = min(mn[1], k1); mx[1] = max(mx[1], k1);
        mn[2] = min(mn[2], k2); mx[2] = max(mx[2], k2);
    }
    for (int a = 0; a < 3; a++) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; a++) {
            atomicMin(&kmin[3 * node + a], mn[a]);
            atomicMax(&kmax[3 * node + a], mx[a]);
        }
    }
}

// Slot bit `pass` of every particle of the chunk's node: axis and mid per
// node; pcnt = per-node part counts after the previous pass (8 per node).
__global__ void k_codes(ChunkArgs c, int pass, const signed char *__restrict__ axis_of, const double *__restrict__ mid,
                        const int *__restrict__ pcnt, const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, unsigned char *__restrict__ code, int *__restrict__ ncnt)
{
    const int ch = blockIdx.x, node = c.chunk_node[ch], b = c.chunk_begin[ch], n = c.chunk_len[ch];
    const int ax = axis_of[3 * node + pass];
    if (ax < 0) return;
    const double *v = ax == 0 ? x : ax == 1 ? y : z;
    const double m = mid[3 * node + ax];
    __shared__ int hist[8];
    if (threadIdx.x < 8) hist[threadIdx.x] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int part = pass == 0 ? 0 : code[b + i];
        int cntp = pcnt[8 * node + part];
        double a = v[b + i];
        int upper = (cntp >= 2) ? !(a <= m) : !(a < m);
        int cd = part | (upper << pass);
        code[b + i] = (unsigned char)cd;
        atomicAdd(&hist[cd], 1);
    }
    __syncthreads();
    if (threadIdx.x < 8 && hist[threadIdx.x]) atomicAdd(&ncnt[8 * node + threadIdx.x], hist[threadIdx.x]);
}

__global__ void k_chunk_hist(ChunkArgs c, const unsigned char *__restrict__ code, int *__restrict__ chunk_cnt)
{
    const int ch = blockIdx.x, b = c.chunk_begin[ch], n = c.chunk_len[ch];
    __shared__ int hist[8];
    if (threadIdx.x < 8) hist[threadIdx.x] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&hist[code[b + i]], 1);
    __syncthreads();
    if (threadIdx.x < 8) chunk_cnt[8 * ch + threadIdx.x] = hist[threadIdx.x];
}

// Stable partition of a chunk into its slots; chunk_off[8*chunk + s] is the
// absolute position of the chunk's first slot-s particle.
__global__ void __launch_bounds__(GT_THREADS)
k_scatter(ChunkArgs c, const int *__restrict__ chunk_off, const unsigned char *__restrict__ code, GtArrays src,
          GtArrays dst)
{
    const int ch = blockIdx.x, b = c.chunk_begin[ch], n = c.chunk_len[ch];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = GT_THREADS / 32;
    __shared__ int wcnt[NW][8], wbase[NW][8], running[8];
    if (threadIdx.x < 8) running[threadIdx.x] = chunk_off[8 * ch + threadIdx.x];
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    for (int base = 0; base < n; base += GT_THREADS) {
        const int i = base + threadIdx.x;
        const bool valid = i < n;
        const int s = valid ? code[b + i] : 255;
        int rank = 0;
        for (int k = 0; k < 8; k++) {
            unsigned m = __ballot_sync(0xffffffffu, s == k);
            if (s == k) rank = __popc(m & lt);
            if (lane == 0) wcnt[warp][k] = __popc(m);
        }
        __syncthreads();
        if (threadIdx.x < 8) {
            int run = running[threadIdx.x];
            for (int w = 0; w < NW; w++) {
                wbase[w][threadIdx.x] = run;
                run += wcnt[w][threadIdx.x];
            }
            running[threadIdx.x] = run;
        }
        __syncthreads();
        if (valid) {
            const int d = wbase[warp][s] + rank;
            dst.x[d] = src.x[b + i];
            dst.y[d] = src.y[b + i];
            dst.z[d] = src.z[b + i];
            if (src.q) dst.q[d] = src.q[b + i];
            dst.order[d] = src.order[b + i];
        }
        __syncthreads();
    }
}

__global__ void k_copy_back(ChunkArgs c, GtArrays src, GtArrays dst)
{
    const int ch = blockIdx.x, b = c.chunk_begin[ch], n = c.chunk_len[ch];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        dst.x[b + i] = src.x[b + i];
        dst.y[b + i] = src.y[b + i];
        dst.z[b + i] = src.z[b + i];
        if (src.q) dst.q[b + i] = src.q[b + i];
        dst.order[b + i] = src.order[b + i];
    }
}

__global__ void k_iota(int n, int *__restrict__ o)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = i;
}

__global__ void k_count_diff(size_t n, const double *__restrict__ a, const double *__restrict__ b,
                             unsigned long long *__restrict__ diff)
{
    unsigned long long d = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        d += (__double_as_longlong(a[i]) != __double_as_longlong(b[i]));
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if ((threadIdx.x & 31) == 0 && d) atomicAdd(diff, d);
}

// Split rule of pc_partition_8 (src/tree/partition.c:178-227), as bt_tree.c.
void divide_axes(double xl, double yl, double zl, int max_nc, int div[3])
{
    double mx = xl; if (mx < yl) mx = yl; if (mx < zl) mx = zl;
    double crit = mx / sqrt(2.0);
    int dx = xl >= crit, dy = yl >= crit, dz = zl >= crit;
    if (max_nc == 4) {
        if (xl < yl && xl < zl) dx = 0;
        if (yl < xl && yl < zl) dy = 0;
        if (zl < xl && zl < yl) dz = 0;
        if (dx + dy + dz == 3) dx = 0;
    }
    if (max_nc == 2) {
        if (xl < yl || xl < zl) dx = 0;
        if (yl < xl || yl < zl) dy = 0;
        if (zl < xl || zl < yl) dz = 0;
        if (dx + dy + dz == 3) { dx = 0; dy = 0; }
        if (dx + dy + dz == 2) {
            if (dx == 0) dy = 0;
            else if (dy == 0) dz = 0;
            else if (dz == 0) dx = 0;
        }
    }
    div[0] = dx; div[1] = dy; div[2] = dz;
}

struct HNode {
    int ibeg, np, level, parent, nchild, child[8];
    double box[6];
};

int preorder(const std::vector<HNode> &nodes, int i, int next, std::vector<int> &pre)
{
    pre[i] = next++;
    for (int k = 0; k < nodes[i].nchild; k++) next = preorder(nodes, nodes[i].child[k], next, pre);
    return next;
}

int g_fail_line = 0;

#define GT_CK(call)                                    \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) {                       \
            g_fail_line = __LINE__;                    \
            return (int)e_;                            \
        }                                              \
    } while (0)

// Nodes of one level: at most 8 per split node of the level above, and a
// split node holds more than maxpar particles.
size_t level_nodes_max(int n, int maxpar, int nsys)
{
    size_t split = (size_t)n / ((size_t)(maxpar > 0 ? maxpar : 1) + 1);
    return std::max((size_t)nsys, std::min((size_t)n, 8 * split + 8)) + 1;
}

}  // namespace

int gpu_tree_fail_line() { return g_fail_line; }

size_t gpu_tree_work_bytes(int n, int maxpar, bool with_q, int nsys)
{
    const size_t L = level_nodes_max(n, maxpar, nsys), C = (size_t)n / GT_CHUNK + L;
    const size_t per = (with_q ? 4 : 3) * sizeof(double) + sizeof(int);
    return per * (size_t)n + (size_t)n            // second copy of the particles, slot codes
           + L * (2 * 3 * 8 + 4 * 8 * 4 + 3 * 8 + 3)  // boxes, part counts, mids, axes
           + C * (3 * 4 + 2 * 8 * 4)              // chunk descriptors, histograms, offsets
           + 24 * 256;
}

int gpu_build_tree(int n, const double *x, const double *y, const double *z, const double *q, int maxpar,
                   GtArrays A, void *work, size_t work_bytes, bt_tree *t, cudaStream_t st, long long *launches)
{
    int64_t off[2] = {0, n};
    return gpu_build_forest(1, off, x, y, z, q, maxpar, A, work, work_bytes, t, st, launches);
}

int gpu_build_forest(int nsys, const int64_t *sys_off, const double *x, const double *y, const double *z,
                     const double *q, int maxpar, GtArrays A, void *work, size_t work_bytes, bt_tree *t,
                     cudaStream_t st, long long *launches)
{
    memset(t, 0, sizeof(*t));
    t->max_depth = 1;
    bt_tree_set_roots(t, nsys);
    const int n = (int)sys_off[nsys];
    if (n <= 0) {
        t->leaf_off = (int *)calloc((size_t)nsys + 1, sizeof(int));
        return 0;
    }
    const bool with_q = q != nullptr;
    if (gpu_tree_work_bytes(n, maxpar, with_q, nsys) > work_bytes) return (int)cudaErrorMemoryAllocation;
    char *p = (char *)work;
    auto take = [&](size_t bytes) { char *r = p; p += (bytes + 255) & ~size_t(255); return (void *)r; };
    GtArrays B;
    B.x = (double *)take(8 * (size_t)n); B.y = (double *)take(8 * (size_t)n); B.z = (double *)take(8 * (size_t)n);
    B.q = with_q ? (double *)take(8 * (size_t)n) : nullptr; B.order = (int *)take(4 * (size_t)n);
    if (!with_q) A.q = nullptr;
    unsigned char *code = (unsigned char *)take((size_t)n);
    const size_t nodes_max = level_nodes_max(n, maxpar, nsys), chunks_max = (size_t)n / GT_CHUNK + nodes_max;
    unsigned long long *kmin = (unsigned long long *)take(3 * 8 * nodes_max);
    unsigned long long *kmax = (unsigned long long *)take(3 * 8 * nodes_max);
    int *cnt[3];
    for (int k = 0; k < 3; k++) cnt[k] = (int *)take(8 * 4 * nodes_max);
    int *cnt0 = (int *)take(8 * 4 * nodes_max);
    double *mid = (double *)take(3 * 8 * nodes_max);
    signed char *axis = (signed char *)take(3 * nodes_max);
    int *c_node = (int *)take(4 * chunks_max), *c_begin = (int *)take(4 * chunks_max), *c_len = (int *)take(4 * chunks_max);
    int *c_hist = (int *)take(8 * 4 * chunks_max), *c_off = (int *)take(8 * 4 * chunks_max);
    ChunkArgs ca{c_node, c_begin, c_len};

    GT_CK(cudaMemcpyAsync(A.x, x, 8 * (size_t)n, cudaMemcpyDefault, st));
    GT_CK(cudaMemcpyAsync(A.y, y, 8 * (size_t)n, cudaMemcpyDefault, st));
    GT_CK(cudaMemcpyAsync(A.z, z, 8 * (size_t)n, cudaMemcpyDefault, st));
    if (with_q) GT_CK(cudaMemcpyAsync(A.q, q, 8 * (size_t)n, cudaMemcpyDefault, st));
    k_iota<<<(n + 255) / 256, 256, 0, st>>>(n, A.order);
    (*launches)++;

    std::vector<HNode> nodes;
    std::vector<int> root_node(nsys, -1);
    for (int k = 0; k < nsys; k++) {
        if (sys_off[k + 1] <= sys_off[k]) continue;
        root_node[k] = (int)nodes.size();
        nodes.push_back(HNode{(int)sys_off[k], (int)(sys_off[k + 1] - sys_off[k]), 0, -1, 0, {0}, {0}});
    }
    int lo = 0, hi = (int)nodes.size(), depth = 1;
    std::vector<int> hc_node, hc_begin, hc_len, hc_off;
    std::vector<unsigned long long> hkmin, hkmax;
    std::vector<int> hcnt, hchist;
    std::vector<double> hmid;
    std::vector<signed char> haxis;
    while (lo < hi) {
        const int L = hi - lo;
        // 1. boxes of the level's nodes
        hc_node.clear(); hc_begin.clear(); hc_len.clear();
        for (int i = 0; i < L; i++) {
            const HNode &nd = nodes[lo + i];
            for (int b = 0; b < nd.np; b += GT_CHUNK) {
                hc_node.push_back(i);
                hc_begin.push_back(nd.ibeg + b);
                hc_len.push_back(std::min(GT_CHUNK, nd.np - b));
            }
        }
        int nch = (int)hc_node.size();
        GT_CK(cudaMemcpyAsync(c_node, hc_node.data(), 4 * (size_t)nch, cudaMemcpyHostToDevice, st));
        GT_CK(cudaMemcpyAsync(c_begin, hc_begin.data(), 4 * (size_t)nch, cudaMemcpyHostToDevice, st));
        GT_CK(cudaMemcpyAsync(c_len, hc_len.data(), 4 * (size_t)nch, cudaMemcpyHostToDevice, st));
        GT_CK(cudaMemsetAsync(kmin, 0xff, 3 * 8 * (size_t)L, st));
        GT_CK(cudaMemsetAsync(kmax, 0x00, 3 * 8 * (size_t)L, st));
        k_boxes<<<nch, GT_THREADS, 0, st>>>(ca, A.x, A.y, A.z, kmin, kmax);
        (*launches)++;
        hkmin.resize(3 * (size_t)L);
        hkmax.resize(3 * (size_t)L);
        GT_CK(cudaMemcpyAsync(hkmin.data(), kmin, 3 * 8 * (size_t)L, cudaMemcpyDeviceToHost, st));
        GT_CK(cudaMemcpyAsync(hkmax.data(), kmax, 3 * 8 * (size_t)L, cudaMemcpyDeviceToHost, st));
        GT_CK(cudaStreamSynchronize(st));
        // 2. split decisions on the host (same arithmetic as bt_tree.c)
        std::vector<int> split;               // level-local indices of nodes to split
        hmid.assign(3 * (size_t)L, 0.0);
        haxis.assign(3 * (size_t)L, -1);
        std::vector<int> naxes(L, 0);
        for (int i = 0; i < L; i++) {
            HNode &nd = nodes[lo + i];
            for (int a = 0; a < 3; a++) {
                nd.box[2 * a] = dkey_inv(hkmin[3 * i + a]);
                nd.box[2 * a + 1] = dkey_inv(hkmax[3 * i + a]);
            }
            if (nd.np <= maxpar) continue;
            double xl = nd.box[1] - nd.box[0], yl = nd.box[3] - nd.box[2], zl = nd.box[5] - nd.box[4];
            int max_nc = (nd.np < 2 * maxpar) ? 2 : (nd.np < 4 * maxpar) ? 4 : 8;
            int div[3];
            divide_axes(xl, yl, zl, max_nc, div);
            int k = 0;
            for (int a = 0; a < 3; a++) {
                hmid[3 * i + a] = (nd.box[2 * a + 1] + nd.box[2 * a]) / 2.0;
                if (div[a]) haxis[3 * i + k++] = (signed char)a;
            }
            naxes[i] = k;
            if (k > 0) split.push_back(i);
        }
        if (split.empty()) break;
        // chunks of the nodes being split
        hc_node.clear(); hc_begin.clear(); hc_len.clear();
        for (int i : split) {
            const HNode &nd = nodes[lo + i];
            for (int b = 0; b < nd.np; b += GT_CHUNK) {
                hc_node.push_back(i);
                hc_begin.push_back(nd.ibeg + b);
                hc_len.push_back(std::min(GT_CHUNK, nd.np - b));
            }
        }
        nch = (int)hc_node.size();
        GT_CK(cudaMemcpyAsync(c_node, hc_node.data(), 4 * (size_t)nch, cudaMemcpyHostToDevice, st));
        GT_CK(cudaMemcpyAsync(c_begin, hc_begin.data(), 4 * (size_t)nch, cudaMemcpyHostToDevice, st));
        GT_CK(cudaMemcpyAsync(c_len, hc_len.data(), 4 * (size_t)nch, cudaMemcpyHostToDevice, st));
        GT_CK(cudaMemcpyAsync(mid, hmid.data(), 3 * 8 * (size_t)L, cudaMemcpyHostToDevice, st));
        GT_CK(cudaMemcpyAsync(axis, haxis.data(), 3 * (size_t)L, cudaMemcpyHostToDevice, st));
        // 3. slot bits, one divided axis per pass
        for (int k = 0; k < 3; k++) GT_CK(cudaMemsetAsync(cnt[k], 0, 8 * 4 * (size_t)L, st));
        // part counts before the first pass: the whole node is one part
        hcnt.assign(8 * (size_t)L, 0);
        for (int i : split) hcnt[8 * i] = nodes[lo + i].np;
        GT_CK(cudaMemcpyAsync(cnt0, hcnt.data(), 8 * 4 * (size_t)L, cudaMemcpyHostToDevice, st));
        for (int k = 0; k < 3; k++) {
            k_codes<<<nch, GT_THREADS, 0, st>>>(ca, k, axis, mid, k == 0 ? cnt0 : cnt[k - 1], A.x, A.y, A.z, code, cnt[k]);
            (*launches)++;
        }
        k_chunk_hist<<<nch, GT_THREADS, 0, st>>>(ca, code, c_hist);
        (*launches)++;
        hchist.resize(8 * (size_t)nch);
        GT_CK(cudaMemcpyAsync(hchist.data(), c_hist, 8 * 4 * (size_t)nch, cudaMemcpyDeviceToHost, st));
        GT_CK(cudaStreamSynchronize(st));
        // 4. child ranges and per-chunk scatter offsets
        std::vector<int> tot(8 * (size_t)L, 0);
        for (int c = 0; c < nch; c++)
            for (int s = 0; s < 8; s++) tot[8 * hc_node[c] + s] += hchist[8 * c + s];
        std::vector<int> start(8 * (size_t)L, 0);
        std::vector<char> degenerate(L, 0);
        for (int i : split) {
            const int bits = naxes[i], nslots = 1 << bits;
            int off = 0;
            for (int key = 0; key < nslots; key++) {
                int s = 0;
                for (int b = 0; b < bits; b++) s |= ((key >> (bits - 1 - b)) & 1) << b;
                start[8 * i + s] = off;
                off += tot[8 * i + s];
            }
            for (int s = 0; s < nslots; s++)
                if (tot[8 * i + s] == nodes[lo + i].np) degenerate[i] = 1;   // kept as a leaf (see bt_tree.c)
        }
        hc_off.resize(8 * (size_t)nch);
        {
            std::vector<int> run(8 * (size_t)L);
            for (int i : split)
                for (int s = 0; s < 8; s++) run[8 * i + s] = nodes[lo + i].ibeg + start[8 * i + s];
            for (int c = 0; c < nch; c++) {
                const int i = hc_node[c];
                for (int s = 0; s < 8; s++) {
                    hc_off[8 * c + s] = run[8 * i + s];
                    run[8 * i + s] += hchist[8 * c + s];
                }
            }
        }
        GT_CK(cudaMemcpyAsync(c_off, hc_off.data(), 8 * 4 * (size_t)nch, cudaMemcpyHostToDevice, st));
        k_scatter<<<nch, GT_THREADS, 0, st>>>(ca, c_off, code, A, B);
        k_copy_back<<<nch, GT_THREADS, 0, st>>>(ca, B, A);
        (*launches) += 2;
        // children (next level)
        for (int i : split) {
            if (degenerate[i]) continue;
            const int nslots = 1 << naxes[i];
            for (int s = 0; s < nslots; s++) {
                if (tot[8 * i + s] == 0) continue;   // empty children are skipped (tree_linked_list.c:266)
                HNode ch{};
                ch.ibeg = nodes[lo + i].ibeg + start[8 * i + s];
                ch.np = tot[8 * i + s];
                ch.level = nodes[lo + i].level + 1;
                ch.parent = lo + i;
                const int idx = (int)nodes.size();
                nodes[lo + i].child[nodes[lo + i].nchild++] = idx;
                nodes.push_back(ch);
                depth = std::max(depth, ch.level + 1);
            }
        }
        lo = hi;
        hi = (int)nodes.size();
    }
    GT_CK(cudaGetLastError());

    // pre-order numbering and the flattened tree (as bt_tree.c)
    const int nn = (int)nodes.size();
    std::vector<int> pre(nn);
    for (int k = 0, next = 0; k < nsys; k++)
        if (root_node[k] >= 0) {
            t->roots[k] = next;
            next = preorder(nodes, root_node[k], next, pre);
        }
    std::vector<HNode> pn(nn);
    for (int i = 0; i < nn; i++) pn[pre[i]] = nodes[i];
    bt_tree_alloc(t, nn);
    t->max_depth = depth;
    for (int k = 0; k < nn; k++) {
        const HNode &nd = pn[k];
        t->ibeg[k] = nd.ibeg; t->numpar[k] = nd.np; t->level[k] = nd.level;
        t->parent[k] = nd.parent >= 0 ? pre[nd.parent] : -1;
        t->nchild[k] = nd.nchild;
        for (int j = 0; j < nd.nchild; j++) t->child[8 * k + j] = pre[nd.child[j]];
        double x0 = nd.box[0], x1 = nd.box[1], y0 = nd.box[2], y1 = nd.box[3], z0 = nd.box[4], z1 = nd.box[5];
        double xl = x1 - x0, yl = y1 - y0, zl = z1 - z0;
        t->x0[k] = x0; t->x1[k] = x1; t->y0[k] = y0; t->y1[k] = y1; t->z0[k] = z0; t->z1[k] = z1;
        t->xm[k] = (x1 + x0) / 2.0; t->ym[k] = (y1 + y0) / 2.0; t->zm[k] = (z1 + z0) / 2.0;
        t->rad[k] = sqrt(xl * xl + yl * yl + zl * zl) / 2.0;
    }
    bt_tree_finish(t);
    return 0;
}

int gpu_arrays_equal(const double *a, const double *b, size_t n, unsigned long long *scratch, bool *equal,
                     cudaStream_t st)
{
    GT_CK(cudaMemsetAsync(scratch, 0, 8, st));
    k_count_diff<<<1184, 256, 0, st>>>(n, a, b, scratch);
    unsigned long long h = 1;
    GT_CK(cudaMemcpyAsync(&h, scratch, 8, cudaMemcpyDeviceToHost, st));
    GT_CK(cudaStreamSynchronize(st));
    *equal = h == 0;
    return 0;
}

}  // namespace bt
