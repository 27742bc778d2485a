// bt_tc.cu -- tensor-core (tcgen05) contractions of barytree_b200.
//
// Leaf P2M of the mixed-precision path as a GEMM on the 5th-generation tensor
// cores.  With Lx, Ly, Lz the barycentric Lagrange bases of a particle on the
// leaf's Chebyshev grid (src/clusters/clusters.c:800-1004),
//   Q[k1, k2, k3] = sum_i (q_i Lx_i[k1]) (Ly_i[k2] Lz_i[k3]),
// i.e. D[m, k1] = sum_i A[m, i] B[k1, i] with m = (k2, k3) (M = (n+1)^2 rows,
// padded to 128), k1 the N dimension (n+1 columns, padded to 16) and the
// leaf's particles the K dimension.  Operands are split into TF32 pairs
// (x = hi + lo) and accumulated as hi*hi + hi*lo + lo*hi in FP32 (3xTF32,
// about FP32 accuracy per product); the accumulator lives in tensor memory.
//
// One CTA per leaf, 128 threads.  Per chunk of 32 particles the threads
// evaluate the bases, form the operands, round them to TF32 pairs and store
// them in shared memory in the canonical K-major layout without swizzling
// (8-row x 16-byte core matrices; the two core matrices of one 8-wide K step
// 128 bytes apart, 8-row groups 256 bytes apart).  Thread 0 issues 12
// tcgen05.mma (4 K steps x 3 products) and commits them to an mbarrier; the
// threads evaluate the next chunk's bases while the tensor core works.
// Bases are FP64 (exact-node rule included), stored as FP32; a product a*b
// splits into hi = tf32(a*b) and the TF32 rounding of the exact FP32 rest
// fma(a, b, -hi).
//
// The tensor core's FP32 accumulation does not round to nearest, so long
// FP32 sums drift (about 1e-6 relative over a 2000-particle leaf): each chunk
// therefore sums into fresh accumulators, hi*hi apart from the small cross
// products, and the threads fold every chunk into FP64 registers (about
// 1.4e-7 relative, a few times the FP32 rounding of the proxies).  Every
// mbarrier wait is bounded: on expiry the kernel records the failure, frees
// its tensor memory and returns without writing.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstdlib>

#include "bt_kernels.cuh"
#include "bt_tc.h"

namespace bt {

namespace {

constexpr int TC_THREADS = 128;
constexpr int TC_M = 128;                  // MMA rows: (k2, k3) pairs, padded
constexpr int TC_N = 16;                   // MMA columns: k1, padded
constexpr int TC_KC = 32;                  // particles per chunk
constexpr int TC_KSTEPS = TC_KC / 8;       // one tcgen05.mma (kind::tf32) covers K = 8
constexpr int TC_MAXNP1 = 16;              // (n+1)^2 <= 256: one or two 128-row tiles
constexpr long long TC_WAIT_LIMIT = 1LL << 22;
constexpr long long TC_TEST_WAIT_LIMIT = 1LL << 10;   // the failure-path test's wait

// Shared-memory layout (bytes).  A tile: 128 rows x 32 tf32; B tile: 16 x 32;
// bases: float [axis][k][particle], rows padded to LSTR floats (16-byte rows
// whose bank groups differ for consecutive k).
constexpr int LSTR = 36;
constexpr uint32_t A_BYTES = TC_M * TC_KC * 4;                  // 16 KB per 128-row tile
constexpr uint32_t B_BYTES = TC_N * TC_KC * 4;                  // 2 KB

// Layout of k_p2m_tc<NP1>: NT = ceil((n+1)^2 / 128) row tiles of A (hi tiles,
// then lo tiles), B [hi, lo], the bases float [3][NP1][LSTR], the grid
// relative to its centre float [3][NP1], the mbarrier and the TMEM address.
template <int NP1>
struct P2mLayout {
    static constexpr int NT = (NP1 * NP1 + TC_M - 1) / TC_M;
    static constexpr uint32_t OFF_A = 0;
    static constexpr uint32_t OFF_B = OFF_A + 2 * NT * A_BYTES;
    static constexpr uint32_t OFF_L = OFF_B + 2 * B_BYTES;
    static constexpr uint32_t OFF_NODES = OFF_L + 3 * NP1 * LSTR * 4;
    static constexpr uint32_t OFF_BAR = (OFF_NODES + 3 * NP1 * 4 + 15) / 16 * 16;
    static constexpr uint32_t OFF_MISC = OFF_BAR + 16;
    static constexpr uint32_t SMEM = OFF_MISC + 16;
    static constexpr uint32_t TMEM_COLS = NT == 1 ? 32 : 64;    // per tile: hi*hi 16 columns, cross products 16
};

// byte offset of element (row, k) of a K-major tile with `rows` rows
__device__ __forceinline__ uint32_t kmajor_off(int rows, int row, int k)
{
    return (uint32_t)((k >> 3) * rows * 32 + (row >> 3) * 256 + ((k >> 2) & 1) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// 1/d in FP32: the MUFU approximation refined by one Newton-Raphson step
// r <- r (2 - d r), which leaves about one ulp of error
__device__ __forceinline__ float rcp_nr(float d)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
    return r * fmaf(-d, r, 2.0f);
}

constexpr uint32_t TF32_MASK = 0xFFFFE000u;     // sign, exponent and the 10 stored mantissa bits of a TF32

// x rounded to the nearest TF32 (ties away from zero): adding half a TF32
// ulp to the magnitude bits and clearing the 13 low bits carries into the
// exponent where the mantissa overflows, as rounding should (finite x well
// below FLT_MAX, as here)
__device__ __forceinline__ uint32_t tf32_round(float x)
{
    return (__float_as_uint(x) + 0x1000u) & TF32_MASK;
}

// p = hi + lo with hi = p rounded to TF32 and lo the rest (exact in FP32),
// also rounded: hi + lo carries p to about 2^-22 relative, without bias (the
// 3xTF32 products hi*hi + hi*lo + lo*hi)
__device__ __forceinline__ void split_tf32(float p, uint32_t &hi, uint32_t &lo)
{
    hi = tf32_round(p);
    lo = tf32_round(p - __uint_as_float(hi));
}

// Shared-memory matrix descriptor: no swizzle, K-major; LBO = distance of the
// two core matrices of one K step, SBO = distance of 8-row groups; bits 46-47
// hold the descriptor version of sm_100.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr)
{
    uint64_t d = (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)(128 >> 4) << 16;
    d |= (uint64_t)(256 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor, kind::tf32: D FP32 (bits 4-5 = 1), A and B TF32
// (bits 7-9 and 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(TC_IDESC), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Bounded wait for the completion of phase `parity` of an mbarrier.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, long long limit = TC_WAIT_LIMIT)
{
    for (long long it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <int NP1>
__global__ void __launch_bounds__(TC_THREADS)
k_p2m_tc(const int *__restrict__ leaves, const int *__restrict__ ibeg, const int *__restrict__ numpar,
         const double *__restrict__ grid, const double *__restrict__ sx, const double *__restrict__ sy,
         const double *__restrict__ sz, const double *__restrict__ sq, double *__restrict__ Q, int *err,
         int expire_test)
{
    using Ly = P2mLayout<NP1>;
    constexpr int n = NP1 - 1, ROWS = NP1 * NP1, P = ROWS * NP1, NT = Ly::NT;
    extern __shared__ __align__(1024) unsigned char sm[];
    float *Lb = reinterpret_cast<float *>(sm + Ly::OFF_L);      // [axis][k][particle], rows of LSTR
    float *nodes = reinterpret_cast<float *>(sm + Ly::OFF_NODES);   // [axis][k], relative to the grid's centre
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + Ly::OFF_BAR);
    uint32_t *misc = reinterpret_cast<uint32_t *>(sm + Ly::OFF_MISC);  // [0] tmem address, [1] status
    unsigned char *Bh = sm + Ly::OFF_B, *Bl = Bh + B_BYTES;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int node = leaves[blockIdx.x];

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(misc)),
                     "r"(Ly::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        misc[1] = 1;
    }
    // each axis's grid relative to its centre, in FP32: the bases are
    // evaluated at FP32 relative coordinates (FP64 difference, rounded once)
    const double *g = grid + (size_t)node * 3 * NP1;
    const double cx = 0.5 * (g[0] + g[n]), cy = 0.5 * (g[NP1] + g[NP1 + n]), cz = 0.5 * (g[2 * NP1] + g[2 * NP1 + n]);
    if (t < 3 * NP1) {
        const int ax = t / NP1;
        nodes[t] = (float)(g[t] - (ax == 0 ? cx : ax == 1 ? cy : cz));
    }
    // operand tiles start zero: padding rows and columns are never written
    for (uint32_t o = t * 16; o < Ly::OFF_L; o += TC_THREADS * 16) *reinterpret_cast<uint4 *>(sm + o) = make_uint4(0, 0, 0, 0);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = misc[0];

    const int b0 = ibeg[node], m = numpar[node];
    const int nch = (m + TC_KC - 1) / TC_KC;
    double acc[NT][NP1];                       // rows t + 128 tile of Q (TMEM lanes), FP64 across chunks
#pragma unroll
    for (int a = 0; a < NT; a++)
#pragma unroll
        for (int k = 0; k < NP1; k++) acc[a][k] = 0.0;
    bool ok = true;
    const uint32_t bar_a = smem_addr(bar);
    if (expire_test) {
        // failure-path test: wait, before any MMA is issued, on a phase that
        // nothing completes; the bounded wait expires and the kernel takes
        // its error exit
        if (t == 0) misc[1] = bar_wait(bar_a, 0u, TC_TEST_WAIT_LIMIT) ? 1u : 0u;
        __syncthreads();
        ok = misc[1] != 0;
    }

    // Bases of one chunk: warp a < 3 evaluates axis a for the chunk's 32
    // particles (lane = particle), barycentric form in FP32 with the
    // exact-node rule on the FP32 relative coordinate; the x bases carry the
    // charge.  Particles past the leaf's end get zero bases.  The coordinate
    // (and charge) of a lane's particle are loaded one chunk ahead, so the
    // global-memory latency overlaps the previous chunk's work.
    const double *src = warp == 0 ? sx : warp == 1 ? sy : sz;
    const double ctr = warp == 0 ? cx : warp == 1 ? cy : cz;
    auto fetch = [&](int c, double &v, double &qv) {
        const int i = c * TC_KC + lane;
        v = 0.0;
        qv = 0.0;
        if (warp < 3 && c < nch && i < m) {
            v = src[b0 + i];
            if (warp == 0) qv = sq[b0 + i];
        }
    };
    auto bases = [&](int c, double v, double qv) {
        if (warp >= 3) return;
        const int i = c * TC_KC + lane;
        float L[NP1];
        if (i < m) {
            const float xr = (float)(v - ctr);
            const float *nd = nodes + warp * NP1;
            float sum = 0.0f;
            int ex = -1;
#pragma unroll
            for (int k = 0; k < NP1; k++) {
                const float d = xr - nd[k];
                if (fabsf(d) < FLT_MIN) ex = k;
                const float w = ((k & 1) ? -1.0f : 1.0f) * ((k == 0 || k == n) ? 0.5f : 1.0f);
                L[k] = w * rcp_nr(d);
                sum += L[k];
            }
            const float qf = warp == 0 ? (float)qv : 1.0f;
            if (ex >= 0) {
#pragma unroll
                for (int k = 0; k < NP1; k++) L[k] = k == ex ? qf : 0.0f;
            } else {
                const float scale = rcp_nr(sum) * qf;
#pragma unroll
                for (int k = 0; k < NP1; k++) L[k] *= scale;
            }
        } else {
#pragma unroll
            for (int k = 0; k < NP1; k++) L[k] = 0.0f;
        }
#pragma unroll
        for (int k = 0; k < NP1; k++) Lb[(warp * NP1 + k) * LSTR + lane] = L[k];
    };

    // chunk c: per tile, hi*hi into accumulator columns 0-15 and the two
    // cross products into columns 16-31 of the tile's 32, from zero (short
    // FP32 sums on the tensor core), folded into FP64 registers once its
    // MMAs have completed.  The next chunk's bases are evaluated while the
    // tensor core works.
    double pv, pq;                 // the next chunk's coordinate and charge (prefetched)
    fetch(0, pv, pq);
    if (ok) bases(0, pv, pq);
    fetch(1, pv, pq);
    __syncthreads();
    for (int c = 0; c < nch && ok; c++) {
        // A rows r = (k2, k3): Ly[k2] * Lz[k3] for the chunk's particles
#pragma unroll
        for (int tile = 0; tile < NT; tile++) {
            const int r = t + TC_M * tile;
            if (r < ROWS) {
                const int k2 = r % NP1, k3 = r / NP1;
                const float *ly = Lb + (1 * NP1 + k2) * LSTR, *lz = Lb + (2 * NP1 + k3) * LSTR;
                unsigned char *Ah = sm + Ly::OFF_A + tile * A_BYTES, *Al = Ah + NT * A_BYTES;
#pragma unroll
                for (int k4 = 0; k4 < TC_KC; k4 += 4) {
                    const float4 a = *reinterpret_cast<const float4 *>(ly + k4);
                    const float4 b = *reinterpret_cast<const float4 *>(lz + k4);
                    uint4 h, l;
                    split_tf32(a.x * b.x, h.x, l.x);
                    split_tf32(a.y * b.y, h.y, l.y);
                    split_tf32(a.z * b.z, h.z, l.z);
                    split_tf32(a.w * b.w, h.w, l.w);
                    const uint32_t o = kmajor_off(TC_M, t, k4);
                    *reinterpret_cast<uint4 *>(Ah + o) = h;
                    *reinterpret_cast<uint4 *>(Al + o) = l;
                }
            }
        }
        {
            // B rows k1: q * Lx[k1]; thread t covers row t / 8, particles 4 (t % 8) .. +3
            const int k1 = t >> 3, k4 = (t & 7) * 4;
            if (k1 < NP1) {
                const float4 a = *reinterpret_cast<const float4 *>(Lb + k1 * LSTR + k4);
                uint4 h, l;
                split_tf32(a.x, h.x, l.x);
                split_tf32(a.y, h.y, l.y);
                split_tf32(a.z, h.z, l.z);
                split_tf32(a.w, h.w, l.w);
                const uint32_t o = kmajor_off(TC_N, k1, k4);
                *reinterpret_cast<uint4 *>(Bh + o) = h;
                *reinterpret_cast<uint4 *>(Bl + o) = l;
            }
        }
        // make the operands visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t bh = smem_addr(Bh), bl = smem_addr(Bl);
#pragma unroll
            for (int tile = 0; tile < NT; tile++) {
                const uint32_t ah = smem_addr(sm + Ly::OFF_A + tile * A_BYTES), al = ah + NT * A_BYTES;
                const uint32_t d = tmem + 32 * tile;
#pragma unroll
                for (int s = 0; s < TC_KSTEPS; s++) {
                    const uint32_t oa = s * TC_M * 32, ob = s * TC_N * 32;
                    mma_tf32(d, smem_desc(ah + oa), smem_desc(bh + ob), s > 0 ? 1u : 0u);
                    mma_tf32(d + 16, smem_desc(ah + oa), smem_desc(bl + ob), s > 0 ? 1u : 0u);
                    mma_tf32(d + 16, smem_desc(al + oa), smem_desc(bh + ob), 1u);
                }
            }
            mma_commit(bar_a);
        }
        // the next chunk's bases (the operands of this chunk are formed)
        if (c + 1 < nch) {
            bases(c + 1, pv, pq);
            fetch(c + 2, pv, pq);
        }
        // this chunk's accumulators, once its MMAs have completed
        const bool done = bar_wait(bar_a, (uint32_t)(c & 1));
        if (done) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int tile = 0; tile < NT; tile++) {
                uint32_t r[32];
                const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + 32 * tile;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                    "[%32];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                      "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                      "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int k = 0; k < NP1; k++)
                    acc[tile][k] += (double)__uint_as_float(r[k]) + (double)__uint_as_float(r[16 + k]);
            }
        }
        // orders the accumulator loads before the next MMAs and the new bases
        // before the next operands; a wait that expired anywhere ends the loop
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        ok = !__syncthreads_or(done ? 0 : 1);
        if (!ok && t == 0) {
            // one more bounded wait for the MMAs in flight before the memory is released
            bar_wait(bar_a, (uint32_t)(c & 1));
        }
    }
    if (ok) {
#pragma unroll
        for (int tile = 0; tile < NT; tile++) {
            const int r = t + TC_M * tile;
            if (r < ROWS) {
#pragma unroll
                for (int k1 = 0; k1 < NP1; k1++) Q[(size_t)node * P + k1 + NP1 * r] = acc[tile][k1];
            }
        }
    } else if (t == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Ly::TMEM_COLS));
    }
}

template <int NP1>
void p2m_tc_t(int nleaves, const int *leaves, const int *ibeg, const int *numpar, const double *grid,
              const double *sx, const double *sy, const double *sz, const double *sq, double *Q, int *err,
              cudaStream_t st)
{
    // BARYTREE_B200_TEST_EXPIRE_TC_WAIT=1 makes every block's first wait run
    // out (no MMA in flight), to test the timeout path end to end
    const int expire_now = getenv("BARYTREE_B200_TEST_EXPIRE_TC_WAIT") != nullptr;
    cudaFuncSetAttribute(k_p2m_tc<NP1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P2mLayout<NP1>::SMEM);
    k_p2m_tc<NP1><<<nleaves, TC_THREADS, P2mLayout<NP1>::SMEM, st>>>(leaves, ibeg, numpar, grid, sx, sy, sz, sq, Q, err,
                                                          expire_now);
}

// ---------------------------------------------------------------------------
// Hermite P2M on the tensor cores (pc_comp_ms_modifiedF_hermite,
// src/clusters/clusters.c:1224-1514): the 8 moments of a node,
//   Q_m[k1, k2, k3] = sum_i q_i X_i[k1] Y_i[k2] Z_i[k3],
// each of X, Y, Z the value basis A or the derivative basis B of its axis
// (m = AAA, BAA, ABA, AAB, BBA, ABB, BAB, BBB in x, y, z), are one GEMM:
// rows (yz pair, k2, k3) of Y*Z for the four pairs AA, BA, AB, BB
// (4 (n+1)^2 <= 256 rows: two M = 128 tiles), columns (x basis, k1) of
// q X for A and B (2 (n+1) <= 16), the particles as K.  Same chunking as
// the FP64 kernels (HermChunk: a node's particles in chunks of up to 2048,
// partial moments summed by k_hermite_reduce) and the same pipeline as
// k_p2m_tc: FP32 bases at FP32 relative coordinates, 3xTF32 products in
// TMEM, folded into FP64 every 32 particles.  Degrees with n + 1 <= 8.
// ---------------------------------------------------------------------------

constexpr int HT_MAXNP1 = 8;
constexpr uint32_t HT_A_TILE = TC_M * TC_KC * 4;                  // 16 KB per 128-row tile
constexpr uint32_t HT_OFF_A = 0;                                  // [tile 0 hi, tile 1 hi, tile 0 lo, tile 1 lo]
constexpr uint32_t HT_OFF_B = HT_OFF_A + 4 * HT_A_TILE;           // [hi, lo]
constexpr uint32_t HT_OFF_L = HT_OFF_B + 2 * B_BYTES;             // float [axis][A/B][k][LSTR]
constexpr uint32_t HT_OFF_NODES = HT_OFF_L + 3 * 2 * HT_MAXNP1 * LSTR * 4;   // float [3][8] nodes, [3][8] w_x
constexpr uint32_t HT_OFF_BAR = (HT_OFF_NODES + 2 * 3 * HT_MAXNP1 * 4 + 15) / 16 * 16;
constexpr uint32_t HT_OFF_MISC = HT_OFF_BAR + 16;
constexpr uint32_t HT_SMEM = HT_OFF_MISC + 16;
constexpr uint32_t HT_TMEM_COLS = 64;                             // per tile: hi*hi 16 columns, cross products 16

template <int NP1>
__global__ void __launch_bounds__(TC_THREADS)
k_p2m_hermite_tc(const HermChunkTc *__restrict__ chunks, const double *__restrict__ grid,
                 const double *__restrict__ box_len, const double *__restrict__ ww, const double *__restrict__ sx,
                 const double *__restrict__ sy, const double *__restrict__ sz, const double *__restrict__ sq,
                 double *__restrict__ Q, double *__restrict__ partial, int *err)
{
    constexpr int n = NP1 - 1, COLS = NP1 * NP1, P = COLS * NP1, ROWS = 4 * COLS, NT = (ROWS + TC_M - 1) / TC_M;
    extern __shared__ __align__(1024) unsigned char sm[];
    float *Lb = reinterpret_cast<float *>(sm + HT_OFF_L);
    float *nodes = reinterpret_cast<float *>(sm + HT_OFF_NODES);    // [3][8]
    float *wx = nodes + 3 * HT_MAXNP1;                               // [3][8]: -4 w_k / len
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + HT_OFF_BAR);
    uint32_t *misc = reinterpret_cast<uint32_t *>(sm + HT_OFF_MISC);
    unsigned char *Bh = sm + HT_OFF_B, *Bl = Bh + B_BYTES;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const HermChunkTc ch = chunks[blockIdx.x];
    const int node = ch.node;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(misc)),
                     "r"(HT_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const double *g = grid + (size_t)node * 3 * NP1;
    const double cx = 0.5 * (g[0] + g[n]), cy = 0.5 * (g[NP1] + g[NP1 + n]), cz = 0.5 * (g[2 * NP1] + g[2 * NP1 + n]);
    if (t < 3 * NP1) {
        const int ax = t / NP1, k = t % NP1;
        nodes[ax * HT_MAXNP1 + k] = (float)(g[t] - (ax == 0 ? cx : ax == 1 ? cy : cz));
        wx[ax * HT_MAXNP1 + k] = (float)(-4.0 * ww[k] / box_len[node * 3 + ax]);
    }
    for (uint32_t o = t * 16; o < HT_OFF_L; o += TC_THREADS * 16) *reinterpret_cast<uint4 *>(sm + o) = make_uint4(0, 0, 0, 0);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = misc[0];
    const int b0 = ch.begin, m = ch.count;
    const int nch = (m + TC_KC - 1) / TC_KC;
    double acc[NT][2 * NP1];
#pragma unroll
    for (int a = 0; a < NT; a++)
#pragma unroll
        for (int c = 0; c < 2 * NP1; c++) acc[a][c] = 0.0;
    const uint32_t bar_a = smem_addr(bar);
    bool ok = true;

    const double *src = warp == 0 ? sx : warp == 1 ? sy : sz;
    const double ctr = warp == 0 ? cx : warp == 1 ? cy : cz;
    auto fetch = [&](int c, double &v, double &qv) {
        const int i = c * TC_KC + lane;
        v = 0.0;
        qv = 0.0;
        if (warp < 3 && c < nch && i < m) {
            v = src[b0 + i];
            if (warp == 0) qv = sq[b0 + i];
        }
    };
    // value (A) and derivative (B) bases of one axis per warp, as
    // hermite_basis (clusters.c:1289-1344) in FP32: A_k = dj/d^2 + wx_k/d,
    // B_k = dj/d, both over sum_j A_j; exact node: A = indicator, B = 0.  The
    // x bases carry the charge.
    auto bases = [&](int c, double v, double qv) {
        if (warp >= 3) return;
        const int i = c * TC_KC + lane;
        float A[NP1], Bv[NP1];
        if (i < m) {
            const float xr = (float)(v - ctr);
            const float *nd = nodes + warp * HT_MAXNP1, *w = wx + warp * HT_MAXNP1;
            float sum = 0.0f;
            int ex = -1;
#pragma unroll
            for (int k = 0; k < NP1; k++) {
                const float d = xr - nd[k];
                if (fabsf(d) < FLT_MIN) ex = k;
                const float r = rcp_nr(d), dj = (k == 0 || k == n) ? 0.25f : 1.0f;
                Bv[k] = dj * r;
                A[k] = r * fmaf(dj, r, w[k]);
                sum += A[k];
            }
            const float qf = warp == 0 ? (float)qv : 1.0f;
            if (ex >= 0) {
#pragma unroll
                for (int k = 0; k < NP1; k++) { A[k] = k == ex ? qf : 0.0f; Bv[k] = 0.0f; }
            } else {
                const float scale = rcp_nr(sum) * qf;
#pragma unroll
                for (int k = 0; k < NP1; k++) { A[k] *= scale; Bv[k] *= scale; }
            }
        } else {
#pragma unroll
            for (int k = 0; k < NP1; k++) A[k] = Bv[k] = 0.0f;
        }
#pragma unroll
        for (int k = 0; k < NP1; k++) {
            Lb[((warp * 2 + 0) * HT_MAXNP1 + k) * LSTR + lane] = A[k];
            Lb[((warp * 2 + 1) * HT_MAXNP1 + k) * LSTR + lane] = Bv[k];
        }
    };

    double pv, pq;
    fetch(0, pv, pq);
    bases(0, pv, pq);
    fetch(1, pv, pq);
    __syncthreads();
    for (int c = 0; c < nch && ok; c++) {
        // A rows r = (pair s, k2, k3): Y_s[k2] Z_s[k3] for the chunk's particles
#pragma unroll
        for (int tile = 0; tile < NT; tile++) {
            const int r = t + TC_M * tile;
            if (r < ROWS) {
                const int sp = r / COLS, col = r % COLS, k2 = col % NP1, k3 = col / NP1;
                const float *ly = Lb + ((1 * 2 + (sp & 1)) * HT_MAXNP1 + k2) * LSTR;
                const float *lz = Lb + ((2 * 2 + (sp >> 1)) * HT_MAXNP1 + k3) * LSTR;
                unsigned char *Ah = sm + HT_OFF_A + tile * HT_A_TILE, *Al = Ah + 2 * HT_A_TILE;
#pragma unroll
                for (int k4 = 0; k4 < TC_KC; k4 += 4) {
                    const float4 a = *reinterpret_cast<const float4 *>(ly + k4);
                    const float4 b = *reinterpret_cast<const float4 *>(lz + k4);
                    uint4 h, l;
                    split_tf32(a.x * b.x, h.x, l.x);
                    split_tf32(a.y * b.y, h.y, l.y);
                    split_tf32(a.z * b.z, h.z, l.z);
                    split_tf32(a.w * b.w, h.w, l.w);
                    const uint32_t o = kmajor_off(TC_M, t, k4);
                    *reinterpret_cast<uint4 *>(Ah + o) = h;
                    *reinterpret_cast<uint4 *>(Al + o) = l;
                }
            }
        }
        {
            // B rows (x basis X, k1): q X[k1]; thread t covers row t / 8, particles 4 (t % 8) .. +3
            const int row = t >> 3, k4 = (t & 7) * 4;
            if (row < 2 * NP1) {
                const int X = row / NP1, k1 = row % NP1;
                const float4 a = *reinterpret_cast<const float4 *>(Lb + ((0 * 2 + X) * HT_MAXNP1 + k1) * LSTR + k4);
                uint4 h, l;
                split_tf32(a.x, h.x, l.x);
                split_tf32(a.y, h.y, l.y);
                split_tf32(a.z, h.z, l.z);
                split_tf32(a.w, h.w, l.w);
                const uint32_t o = kmajor_off(TC_N, row, k4);
                *reinterpret_cast<uint4 *>(Bh + o) = h;
                *reinterpret_cast<uint4 *>(Bl + o) = l;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t bh = smem_addr(Bh), bl = smem_addr(Bl);
#pragma unroll
            for (int tile = 0; tile < NT; tile++) {
                const uint32_t ah = smem_addr(sm + HT_OFF_A + tile * HT_A_TILE), al = ah + 2 * HT_A_TILE;
                const uint32_t d = tmem + 32 * tile;
#pragma unroll
                for (int s = 0; s < TC_KSTEPS; s++) {
                    const uint32_t oa = s * TC_M * 32, ob = s * TC_N * 32;
                    mma_tf32(d, smem_desc(ah + oa), smem_desc(bh + ob), s > 0 ? 1u : 0u);
                    mma_tf32(d + 16, smem_desc(ah + oa), smem_desc(bl + ob), s > 0 ? 1u : 0u);
                    mma_tf32(d + 16, smem_desc(al + oa), smem_desc(bh + ob), 1u);
                }
            }
            mma_commit(bar_a);
        }
        if (c + 1 < nch) {
            bases(c + 1, pv, pq);
            fetch(c + 2, pv, pq);
        }
        const bool done = bar_wait(bar_a, (uint32_t)(c & 1));
        if (done) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int tile = 0; tile < NT; tile++) {
                uint32_t r[32];
                const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + 32 * tile;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                    "[%32];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                      "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                      "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int k = 0; k < 2 * NP1; k++)
                    acc[tile][k] += (double)__uint_as_float(r[k]) + (double)__uint_as_float(r[16 + k]);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        ok = !__syncthreads_or(done ? 0 : 1);
        if (!ok && t == 0) bar_wait(bar_a, (uint32_t)(c & 1));
    }
    if (ok) {
        // moment of (yz pair s, x basis X): AA -> AAA, BAA; BA -> ABA, BBA;
        // AB -> AAB, BAB; BB -> ABB, BBB
        constexpr int MOM[4][2] = {{0, 1}, {2, 4}, {3, 6}, {5, 7}};
        double *dst = ch.slot < 0 ? Q + (size_t)node * 8 * P : partial + (size_t)ch.slot * 8 * P;
#pragma unroll
        for (int tile = 0; tile < NT; tile++) {
            const int r = t + TC_M * tile;
            if (r < ROWS) {
                const int sp = r / COLS, col = r % COLS;
#pragma unroll
                for (int k = 0; k < 2 * NP1; k++)
                    dst[(size_t)MOM[sp][k / NP1] * P + (k % NP1) + NP1 * col] = acc[tile][k];
            }
        }
    } else if (t == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(HT_TMEM_COLS));
    }
}

// ---------------------------------------------------------------------------
// L2P on the tensor cores (cp_comp_pot, src/interaction_compute/
// interaction_compute_downpass.c:326-497): the potential of target i from its
// leaf's grid values Phi[k1, k2, k3] is
//   phi_i = sum_{k2,k3} Ly_i[k2] Lz_i[k3] G[i, (k2, k3)],
//   G[i, (k2, k3)] = sum_k1 Lx_i[k1] Phi[k1, (k2, k3)],
// G a GEMM with the item's 128 targets as M, the (k2, k3) pairs as N (padded
// to 128) and k1 as K (padded to 16): 2 K steps x 3 products (3xTF32) into
// 128 TMEM columns.  Each thread (= TMEM lane = target) then reads its row
// and finishes the (n+1)^2-term contraction in FP32 registers, so the
// (n+1)^3 multiply-adds per target run on the tensor core.
// ---------------------------------------------------------------------------

constexpr int L2_M = 128, L2_N = 128, L2_K = 16;
constexpr int L2_MAXNP1 = 11;                           // (n+1)^2 <= 128 = N
constexpr uint32_t L2_TMEM_COLS = 128;
constexpr uint32_t L2_A_BYTES = L2_M * L2_K * 4;        // 8 KB
constexpr uint32_t L2_B_BYTES = L2_N * L2_K * 4;        // 8 KB
constexpr uint32_t L2_OFF_A = 0;                        // [hi, lo]
constexpr uint32_t L2_OFF_B = L2_OFF_A + 2 * L2_A_BYTES;  // [hi, lo]
constexpr uint32_t L2_OFF_NODES = L2_OFF_B + 2 * L2_B_BYTES;   // float [3][L2_MAXNP1]
constexpr uint32_t L2_OFF_BAR = (L2_OFF_NODES + 3 * L2_MAXNP1 * 4 + 15) / 16 * 16;
constexpr uint32_t L2_OFF_MISC = L2_OFF_BAR + 16;
constexpr uint32_t L2_SMEM = L2_OFF_MISC + 16;
constexpr uint32_t L2_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(L2_N >> 3) << 17) |
                              ((uint32_t)(L2_M >> 4) << 24);

__device__ __forceinline__ void mma_tf32_l2(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(L2_IDESC), "r"(accumulate));
}

// Barycentric Lagrange basis in FP32 at a coordinate relative to the grid's
// centre, with the exact-node rule (the FP32 difference is zero).
template <int NP1>
__device__ __forceinline__ void basis_f32(float xr, const float *nd, float *L)
{
    constexpr int n = NP1 - 1;
    float sum = 0.0f;
    int ex = -1;
#pragma unroll
    for (int k = 0; k < NP1; k++) {
        const float d = xr - nd[k];
        if (fabsf(d) < FLT_MIN) ex = k;
        const float w = ((k & 1) ? -1.0f : 1.0f) * ((k == 0 || k == n) ? 0.5f : 1.0f);
        L[k] = w * rcp_nr(d);
        sum += L[k];
    }
    if (ex >= 0) {
#pragma unroll
        for (int k = 0; k < NP1; k++) L[k] = k == ex ? 1.0f : 0.0f;
    } else {
        const float inv = rcp_nr(sum);
#pragma unroll
        for (int k = 0; k < NP1; k++) L[k] *= inv;
    }
}

template <int NP1>
__global__ void __launch_bounds__(TC_THREADS)
k_l2p_tc(const int2 *__restrict__ items, const int *__restrict__ leaf_node, const int *__restrict__ t_ibeg,
         const int *__restrict__ t_numpar, const double *__restrict__ t_grid, const double *__restrict__ Phi,
         const double *__restrict__ tx, const double *__restrict__ ty, const double *__restrict__ tz,
         double *__restrict__ pot, int *err)
{
    constexpr int n = NP1 - 1, ROWS = NP1 * NP1, P = ROWS * NP1;
    extern __shared__ __align__(1024) unsigned char sm[];
    float *nodes = reinterpret_cast<float *>(sm + L2_OFF_NODES);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L2_OFF_BAR);
    uint32_t *misc = reinterpret_cast<uint32_t *>(sm + L2_OFF_MISC);
    unsigned char *Ah = sm + L2_OFF_A, *Al = Ah + L2_A_BYTES, *Bh = sm + L2_OFF_B, *Bl = Bh + L2_B_BYTES;
    const int t = threadIdx.x, warp = t >> 5;
    const int2 it = items[blockIdx.x];
    const int node = leaf_node[it.x];

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(misc)),
                     "r"(L2_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const double *g = t_grid + (size_t)node * 3 * NP1;
    const double cx = 0.5 * (g[0] + g[n]), cy = 0.5 * (g[NP1] + g[NP1 + n]), cz = 0.5 * (g[2 * NP1] + g[2 * NP1 + n]);
    if (t < 3 * NP1) {
        const int ax = t / NP1;
        nodes[t] = (float)(g[t] - (ax == 0 ? cx : ax == 1 ? cy : cz));
    }
    // B rows (k2, k3): the grid values over k1, split into TF32 pairs; rows
    // and columns past the grid stay zero
    {
        uint32_t h[L2_K], l[L2_K];
#pragma unroll
        for (int k = 0; k < L2_K; k++) h[k] = l[k] = 0u;
        if (t < ROWS) {
#pragma unroll
            for (int k1 = 0; k1 < NP1; k1++) split_tf32((float)Phi[(size_t)node * P + k1 + NP1 * t], h[k1], l[k1]);
        }
#pragma unroll
        for (int k4 = 0; k4 < L2_K; k4 += 4) {
            const uint32_t o = kmajor_off(L2_N, t, k4);
            *reinterpret_cast<uint4 *>(Bh + o) = make_uint4(h[k4], h[k4 + 1], h[k4 + 2], h[k4 + 3]);
            *reinterpret_cast<uint4 *>(Bl + o) = make_uint4(l[k4], l[k4 + 1], l[k4 + 2], l[k4 + 3]);
        }
    }
    __syncthreads();
    // A row t: this target's Lx, split; its Ly and Lz stay in registers
    const int ti = it.y * TC_THREADS + t;
    const bool active = ti < t_numpar[node];
    const int gi = t_ibeg[node] + (active ? ti : 0);
    float Ly[NP1], Lz[NP1];
    {
        float Lx[NP1];
        if (active) {
            basis_f32<NP1>((float)(tx[gi] - cx), nodes, Lx);
            basis_f32<NP1>((float)(ty[gi] - cy), nodes + NP1, Ly);
            basis_f32<NP1>((float)(tz[gi] - cz), nodes + 2 * NP1, Lz);
        } else {
#pragma unroll
            for (int k = 0; k < NP1; k++) Lx[k] = Ly[k] = Lz[k] = 0.0f;
        }
        uint32_t h[L2_K], l[L2_K];
#pragma unroll
        for (int k = 0; k < L2_K; k++) h[k] = l[k] = 0u;
#pragma unroll
        for (int k1 = 0; k1 < NP1; k1++) split_tf32(Lx[k1], h[k1], l[k1]);
#pragma unroll
        for (int k4 = 0; k4 < L2_K; k4 += 4) {
            const uint32_t o = kmajor_off(L2_M, t, k4);
            *reinterpret_cast<uint4 *>(Ah + o) = make_uint4(h[k4], h[k4 + 1], h[k4 + 2], h[k4 + 3]);
            *reinterpret_cast<uint4 *>(Al + o) = make_uint4(l[k4], l[k4 + 1], l[k4 + 2], l[k4 + 3]);
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    const uint32_t tmem = misc[0];
    const uint32_t bar_a = smem_addr(bar);
    if (t == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t ah = smem_addr(Ah), al = smem_addr(Al), bh = smem_addr(Bh), bl = smem_addr(Bl);
        constexpr int KSTEPS = (NP1 + 7) / 8;
#pragma unroll
        for (int s = 0; s < KSTEPS; s++) {
            const uint32_t oa = s * L2_M * 32, ob = s * L2_N * 32;
            mma_tf32_l2(tmem, smem_desc(ah + oa), smem_desc(bh + ob), s > 0 ? 1u : 0u);
            mma_tf32_l2(tmem, smem_desc(ah + oa), smem_desc(bl + ob), 1u);
            mma_tf32_l2(tmem, smem_desc(al + oa), smem_desc(bh + ob), 1u);
        }
        mma_commit(bar_a);
    }
    const bool done = bar_wait(bar_a, 0u);
    const bool ok = !__syncthreads_or(done ? 0 : 1);
    if (ok) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float s3[NP1];
#pragma unroll
        for (int k = 0; k < NP1; k++) s3[k] = 0.0f;
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int c0 = 0; c0 < ROWS; c0 += 32) {
            uint32_t r[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                "[%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < 32; j++) {
                const int c = c0 + j;
                if (c < ROWS) s3[c / NP1] = fmaf(Ly[c % NP1], __uint_as_float(r[j]), s3[c / NP1]);
            }
        }
        float phi = 0.0f;
#pragma unroll
        for (int k3 = 0; k3 < NP1; k3++) phi = fmaf(Lz[k3], s3[k3], phi);
        if (active) pot[gi] += (double)phi;
    } else if (t == 0) {
        atomicExch(err, 1);
        bar_wait(bar_a, 0u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L2_TMEM_COLS));
    }
}

template <int NP1>
void l2p_tc_t(int nitems, const int2 *items, const int *leaf_node, const int *t_ibeg, const int *t_numpar,
              const double *t_grid, const double *Phi, const double *tx, const double *ty, const double *tz,
              double *pot, int *err, cudaStream_t st)
{
    cudaFuncSetAttribute(k_l2p_tc<NP1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L2_SMEM);
    k_l2p_tc<NP1><<<nitems, TC_THREADS, L2_SMEM, st>>>(items, leaf_node, t_ibeg, t_numpar, t_grid, Phi, tx, ty, tz,
                                                         pot, err);
}

// ---------------------------------------------------------------------------
// Inference of the degree selector's MLP (6 -> 64 -> 64 -> 64 -> 11, tanh)
// on the tensor cores: every layer of a tile of 128 rows is one GEMM,
// D[row, o] = sum_i A[row, i] W[i, o], with the rows as M = 128, the layer's
// outputs as N (64, or 16 for the 11 outputs) and its inputs as K (8 for the
// 6 features, else 64), 3xTF32 into TMEM.  Each thread (= TMEM lane = row)
// reads its row, adds the bias, applies tanh and writes the next layer's A
// operand.  The weights, split into TF32 pairs, sit in shared memory as the
// B operands for the whole kernel; the two warpgroups of a CTA work on
// different tiles (their own A buffers, mbarriers and TMEM columns), so one's
// MMAs overlap the other's activations.  The network is the one the
// training kernels of bt_learned.cu (k_linear_fwd) evaluate; the sums are
// the tensor core's, so the predictions agree with theirs to FP32 rounding
// (about 1e-6 relative), not bit for bit.
// ---------------------------------------------------------------------------

constexpr int MT_IN = 6, MT_H = 64, MT_OUT = 11, MT_NOUT = 16, MT_K1 = 8;
constexpr uint32_t MT_W1 = 0;                                     // [hi, lo]: N = 64 x K = 8
constexpr uint32_t MT_W1B = MT_H * MT_K1 * 4;                     // 2 KB
constexpr uint32_t MT_W2 = MT_W1 + 2 * MT_W1B;                    // [hi, lo]: 64 x 64
constexpr uint32_t MT_WHB = MT_H * MT_H * 4;                      // 16 KB
constexpr uint32_t MT_W3 = MT_W2 + 2 * MT_WHB;
constexpr uint32_t MT_W4 = MT_W3 + 2 * MT_WHB;                    // [hi, lo]: 16 x 64
constexpr uint32_t MT_W4B = MT_NOUT * MT_H * 4;                   // 4 KB
constexpr uint32_t MT_A = MT_W4 + 2 * MT_W4B;                     // per warpgroup [hi, lo]: 128 x 64
constexpr uint32_t MT_AB = TC_M * MT_H * 4;                       // 32 KB
constexpr uint32_t MT_PAR = MT_A + 2 * 2 * MT_AB;                 // floats: b1 b2 b3 [64], b4 [16], mean, std [6]
constexpr uint32_t MT_NPAR = 3 * MT_H + MT_NOUT + 2 * MT_IN;
constexpr uint32_t MT_BAR = (MT_PAR + MT_NPAR * 4 + 15) / 16 * 16;   // 2 mbarriers, then the TMEM address
constexpr uint32_t MT_SMEM = MT_BAR + 32;
constexpr uint32_t MT_TMEM_COLS = 128;                            // warpgroup w: columns 64 w .. 64 w + 63
__host__ __device__ constexpr uint32_t mt_idesc(int n)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32_n(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// 1 if any of the 128 threads of named barrier `id` passes a nonzero flag
__device__ __forceinline__ int wg_any(int flag, int id)
{
    int r;
    asm volatile(
        "{\n\t"
        ".reg .pred p, q;\n\t"
        "setp.ne.b32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, 128, p;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t"
        "}\n"
        : "=r"(r)
        : "r"(flag), "r"(id)
        : "memory");
    return r;
}

// the B operand of one layer: W[i][o] (I x O, row-major) as N = o rows, K = i
// columns, K-major, zero past I and O, split into TF32 pairs
__device__ void mt_weights(const float *W, int I, int O, int N, int K, unsigned char *hi, unsigned char *lo)
{
    for (int e = threadIdx.x; e < N * K; e += blockDim.x) {
        const int o = e / K, i = e % K;
        const float v = (o < O && i < I) ? W[i * O + o] : 0.0f;
        uint32_t h, l;
        split_tf32(v, h, l);
        const uint32_t off = kmajor_off(N, o, i);
        *reinterpret_cast<uint32_t *>(hi + off) = h;
        *reinterpret_cast<uint32_t *>(lo + off) = l;
    }
}

__global__ void __launch_bounds__(2 * TC_THREADS, 1)
k_mlp_infer_tc(const float *__restrict__ w, int64_t B, const float *__restrict__ X, float *__restrict__ Y, int *err)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    float *par = reinterpret_cast<float *>(sm + MT_PAR);
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + MT_BAR);
    uint32_t *misc = reinterpret_cast<uint32_t *>(sm + MT_BAR + 16);
    const int tid = threadIdx.x, wg = tid >> 7, t = tid & 127, warp = tid >> 5;
    // weight layout of bt_learned.h: norm (mean[6], std[6]), W1[6][64], b1,
    // W2[64][64], b2, W3[64][64], b3, W4[64][11], b4
    const float *norm = w, *W1 = w + 2 * MT_IN, *b1 = W1 + MT_IN * MT_H, *W2 = b1 + MT_H, *b2 = W2 + MT_H * MT_H,
                *W3 = b2 + MT_H, *b3 = W3 + MT_H * MT_H, *W4 = b3 + MT_H, *b4 = W4 + MT_H * MT_OUT;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(misc)),
                     "r"(MT_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bars)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bars + 1)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    mt_weights(W1, MT_IN, MT_H, MT_H, MT_K1, sm + MT_W1, sm + MT_W1 + MT_W1B);
    mt_weights(W2, MT_H, MT_H, MT_H, MT_H, sm + MT_W2, sm + MT_W2 + MT_WHB);
    mt_weights(W3, MT_H, MT_H, MT_H, MT_H, sm + MT_W3, sm + MT_W3 + MT_WHB);
    mt_weights(W4, MT_H, MT_OUT, MT_NOUT, MT_H, sm + MT_W4, sm + MT_W4 + MT_W4B);
    for (int i = tid; i < (int)MT_NPAR; i += blockDim.x) {
        float v;
        if (i < 3 * MT_H) v = (i < MT_H ? b1 : i < 2 * MT_H ? b2 : b3)[i % MT_H];
        else if (i < 3 * MT_H + MT_NOUT) v = i - 3 * MT_H < MT_OUT ? b4[i - 3 * MT_H] : 0.0f;
        else v = norm[i - 3 * MT_H - MT_NOUT];
        par[i] = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = misc[0] + 64 * wg;
    const uint32_t tlane = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    unsigned char *Ah = sm + MT_A + wg * 2 * MT_AB, *Al = Ah + MT_AB;
    const uint32_t bar = smem_addr(bars + wg);
    const int bid = 1 + wg;                            // the warpgroup's named barrier
    const float *bb1 = par, *bb2 = par + MT_H, *bb3 = par + 2 * MT_H, *bb4 = par + 3 * MT_H;
    const float *mean = par + 3 * MT_H + MT_NOUT, *sdev = mean + MT_IN;
    uint32_t phase = 0;
    bool ok = true;

    // one layer: thread 0 of the warpgroup issues the MMAs, all wait for them
    auto layer = [&](uint32_t wofs, uint32_t wbytes, int n, int ksteps) -> bool {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("bar.sync %0, 128;" ::"r"(bid) : "memory");
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ah = smem_addr(Ah), al = smem_addr(Al);
            const uint32_t bh = smem_addr(sm + wofs), bl = bh + wbytes;
            const uint32_t idesc = mt_idesc(n);
            for (int s = 0; s < ksteps; s++) {
                const uint32_t oa = s * TC_M * 32, ob = s * n * 32;
                mma_tf32_n(tmem, smem_desc(ah + oa), smem_desc(bh + ob), idesc, s > 0 ? 1u : 0u);
                mma_tf32_n(tmem, smem_desc(ah + oa), smem_desc(bl + ob), idesc, 1u);
                mma_tf32_n(tmem, smem_desc(al + oa), smem_desc(bh + ob), idesc, 1u);
            }
            mma_commit(bar);
        }
        const bool done = bar_wait(bar, phase);
        phase ^= 1u;
        const bool fail = wg_any(done ? 0 : 1, bid) != 0;
        if (!fail) asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        return !fail;
    };
    // this thread's row of a 64-column layer output, bias and tanh, as the
    // next layer's A operand
    auto activate = [&](const float *bias) {
#pragma unroll
        for (int c0 = 0; c0 < MT_H; c0 += 32) {
            uint32_t r[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                "[%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(tlane + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int k4 = 0; k4 < 32; k4 += 4) {
                uint4 h, l;
                split_tf32(tanhf(__uint_as_float(r[k4]) + bias[c0 + k4]), h.x, l.x);
                split_tf32(tanhf(__uint_as_float(r[k4 + 1]) + bias[c0 + k4 + 1]), h.y, l.y);
                split_tf32(tanhf(__uint_as_float(r[k4 + 2]) + bias[c0 + k4 + 2]), h.z, l.z);
                split_tf32(tanhf(__uint_as_float(r[k4 + 3]) + bias[c0 + k4 + 3]), h.w, l.w);
                const uint32_t o = kmajor_off(TC_M, t, c0 + k4);
                *reinterpret_cast<uint4 *>(Ah + o) = h;
                *reinterpret_cast<uint4 *>(Al + o) = l;
            }
        }
    };

    const int64_t ntiles = (B + TC_M - 1) / TC_M;
    for (int64_t tile = (int64_t)blockIdx.x * 2 + wg; tile < ntiles && ok; tile += (int64_t)gridDim.x * 2) {
        const int64_t row = tile * TC_M + t;
        // layer 1's A: the normalised features, K = 8
        {
            uint4 h = make_uint4(0, 0, 0, 0), l = make_uint4(0, 0, 0, 0), h2 = h, l2 = l;
            uint32_t hv[MT_K1] = {}, lv[MT_K1] = {};
            if (row < B) {
#pragma unroll
                for (int i = 0; i < MT_IN; i++)
                    split_tf32(fminf(fmaxf((X[row * MT_IN + i] - mean[i]) / sdev[i], -4.f), 4.f), hv[i], lv[i]);
            }
            h = make_uint4(hv[0], hv[1], hv[2], hv[3]); h2 = make_uint4(hv[4], hv[5], hv[6], hv[7]);
            l = make_uint4(lv[0], lv[1], lv[2], lv[3]); l2 = make_uint4(lv[4], lv[5], lv[6], lv[7]);
            *reinterpret_cast<uint4 *>(Ah + kmajor_off(TC_M, t, 0)) = h;
            *reinterpret_cast<uint4 *>(Ah + kmajor_off(TC_M, t, 4)) = h2;
            *reinterpret_cast<uint4 *>(Al + kmajor_off(TC_M, t, 0)) = l;
            *reinterpret_cast<uint4 *>(Al + kmajor_off(TC_M, t, 4)) = l2;
        }
        if (!(ok = layer(MT_W1, MT_W1B, MT_H, 1))) break;
        activate(bb1);
        if (!(ok = layer(MT_W2, MT_WHB, MT_H, MT_H / 8))) break;
        activate(bb2);
        if (!(ok = layer(MT_W3, MT_WHB, MT_H, MT_H / 8))) break;
        activate(bb3);
        if (!(ok = layer(MT_W4, MT_W4B, MT_NOUT, MT_H / 8))) break;
        {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(tlane));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < B) {
#pragma unroll
                for (int o = 0; o < MT_OUT; o++) Y[row * MT_OUT + o] = __uint_as_float(r[o]) + bb4[o];
            }
        }
        // the next tile's first MMAs overwrite these columns after the
        // warpgroup's next barrier, which orders the loads above before them
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    if (!ok && t == 0) {
        atomicExch(err, 1);
        bar_wait(bar, phase ^ 1u);          // one more bounded wait for the MMAs in flight
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(misc[0]), "r"(MT_TMEM_COLS));
    }
}

}  // namespace

bool p2m_tc_supported(int n) { return n >= 1 && n + 1 <= TC_MAXNP1; }

bool l2p_tc_supported(int n) { return n >= 1 && n + 1 <= L2_MAXNP1; }

void launch_p2m_tc(int n, int nleaves, const int *leaves, const int *ibeg, const int *numpar, const double *grid,
                   const double *sx, const double *sy, const double *sz, const double *sq, double *Q, int *err,
                   cudaStream_t st)
{
    if (nleaves <= 0) return;
    switch (n + 1) {
#define BT_TC(N) case N: p2m_tc_t<N>(nleaves, leaves, ibeg, numpar, grid, sx, sy, sz, sq, Q, err, st); return;
        BT_TC(2) BT_TC(3) BT_TC(4) BT_TC(5) BT_TC(6) BT_TC(7) BT_TC(8) BT_TC(9) BT_TC(10) BT_TC(11) BT_TC(12)
        BT_TC(13) BT_TC(14) BT_TC(15) BT_TC(16)
#undef BT_TC
    }
}

void launch_l2p_tc(int n, int nitems, const int2 *items, const int *leaf_node, const int *t_ibeg,
                   const int *t_numpar, const double *t_grid, const double *Phi, const double *tx, const double *ty,
                   const double *tz, double *pot, int *err, cudaStream_t st)
{
    if (nitems <= 0) return;
    switch (n + 1) {
#define BT_L2(N) case N: l2p_tc_t<N>(nitems, items, leaf_node, t_ibeg, t_numpar, t_grid, Phi, tx, ty, tz, pot, err, st); return;
        BT_L2(2) BT_L2(3) BT_L2(4) BT_L2(5) BT_L2(6) BT_L2(7) BT_L2(8) BT_L2(9) BT_L2(10) BT_L2(11)
#undef BT_L2
    }
}

bool p2m_hermite_tc_supported(int n) { return n >= 1 && n + 1 <= HT_MAXNP1; }

void launch_p2m_hermite_tc(int n, int nchunks, const HermChunkTc *chunks, const double *grid, const double *box_len,
                           const double *ww, const double *sx, const double *sy, const double *sz, const double *sq,
                           double *Q, double *partial, int *err, cudaStream_t st)
{
    if (nchunks <= 0) return;
    switch (n + 1) {
#define BT_HT(N)                                                                                                       \
    case N:                                                                                                            \
        cudaFuncSetAttribute(k_p2m_hermite_tc<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HT_SMEM);         \
        k_p2m_hermite_tc<N><<<nchunks, TC_THREADS, HT_SMEM, st>>>(chunks, grid, box_len, ww, sx, sy, sz, sq, Q, partial, \
                                                                  err);                                               \
        return;
        BT_HT(2) BT_HT(3) BT_HT(4) BT_HT(5) BT_HT(6) BT_HT(7) BT_HT(8)
#undef BT_HT
    }
}

void mlp_infer_tc(const float *w, int64_t B, const float *X, float *Y, int *err, cudaStream_t st)
{
    if (B <= 0) return;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t pairs = ((B + TC_M - 1) / TC_M + 1) / 2;
    const int grid = (int)std::min<int64_t>(pairs, (int64_t)sms);
    cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MT_SMEM);
    k_mlp_infer_tc<<<grid, 2 * TC_THREADS, MT_SMEM, st>>>(w, B, X, Y, err);
}

}  // namespace bt
