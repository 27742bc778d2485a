// bt_api.cu -- C ABI of barytree_b200 and the per-call driver.
//
// Call flow (mirrors treedriver, src/drivers/treedriver.c:39-1145):
//   host:   validate + params (RunParams_Setup) -> trees/batches -> MAC lists
//           -> device work lists (bt_lists.c)
//   device: upload -> upward pass (P2M, M2M | Hermite P2M) -> grid-output
//           evaluation (M2L + CP) -> L2L -> particle-output evaluation
//           (PC + PP) -> L2P -> download
//   host:   scatter potentials back to the caller's order
//           (Particles_Targets_Reorder, src/particles/particles.c:58-94)
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <climits>
#include <cstring>
#include <future>
#include <mutex>
#include <omp.h>
#include <sys/resource.h>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/barytree_b200.h"
#include "bt_device.h"
#include "bt_mixed.h"
#include "bt_learned.h"
#include "bt_gputree.h"
#include "bt_gpulists.h"
#include "bt_ss.h"
#include "bt_tc.h"
#include "bt_sym.h"
#include "bt_host.h"

namespace {

thread_local char g_err[512] = "";
std::atomic<long long> g_launches{0};

void set_err(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

double now_ms()
{
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Host-side phase times on stderr when the environment variable
// BARYTREE_B200_TIMING is set (diagnostics; device phases are in bt_report).
long minor_faults()
{
    struct rusage ru;
    return getrusage(RUSAGE_SELF, &ru) == 0 ? ru.ru_minflt : 0;
}

struct PhaseTimer {
    bool on;
    double t;
    long flt;
    PhaseTimer() : on(getenv("BARYTREE_B200_TIMING") != nullptr), t(now_ms()), flt(on ? minor_faults() : 0)
    {
        static bool said = false;
        if (on && !said) {
            said = true;
            fprintf(stderr, "[barytree_b200] host threads (OpenMP) %d\n", omp_get_max_threads());
        }
    }
    void mark(const char *what)
    {
        if (!on) return;
        const double n = now_ms();
        const long f = minor_faults();
        fprintf(stderr, "[barytree_b200] %-34s %9.3f ms %8ld page faults\n", what, n - t, f - flt);
        t = n;
        flt = f;
    }
};

// Host vectors whose elements are left uninitialised on construction and
// resize (trivial types): the planning passes write every element they read,
// in parallel, instead of a serial zero fill of tens of MB per call.
template <typename T>
struct NoInit : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = NoInit<U>;
    };
    NoInit() = default;
    template <typename U>
    NoInit(const NoInit<U> &) noexcept {}
    template <typename U>
    void construct(U *p) noexcept(std::is_nothrow_default_constructible<U>::value)
    {
        ::new (static_cast<void *>(p)) U;
    }
    template <typename U, typename... Args>
    void construct(U *p, Args &&...args)
    {
        ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...);
    }
};
template <typename T>
using hvec = std::vector<T, NoInit<T>>;

// Grow-only device arena per device, reused across calls so steady-state
// calls do not touch cudaMalloc.
struct Arena {
    char *base = nullptr;
    size_t cap = 0, used = 0;
    bool fixed = false;     // wraps caller-provided memory: never grows, never frees
    bool reserve(size_t bytes)
    {
        if (bytes <= cap) return true;
        if (fixed) return false;
        if (base) cudaFree(base);
        base = nullptr;
        cap = 0;
        if (cudaMalloc(&base, bytes) != cudaSuccess) { cudaGetLastError(); return false; }
        cap = bytes;
        return true;
    }
    void *take(size_t bytes)
    {
        size_t a = (used + 255) & ~size_t(255);
        used = a + bytes;
        return base + a;
    }
};

// A second stream and its fork / join events: work that is independent of
// the main stream's next kernels runs beside them.
struct Fork {
    cudaStream_t side = nullptr, side2 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, join2 = nullptr;
};

struct DeviceCtx {
    int device = -1;
    cudaStream_t stream = nullptr;
    Fork fk;
    Arena arena;
    Arena tree_arena;       // particles in tree order (GPU tree build), kept through the call
    cudaEvent_t ev[8] = {};
    std::mutex mu;
};

DeviceCtx g_ctx[16];
std::mutex g_ctx_mu;

// Per-call choices that shape the device sequence: tile shape and dispatch
// of the mixed particle-output kernel, the upward-pass kernel, and the
// share of the target leaves this call evaluates.
struct EvalConfig {
    bool queue = false;
    int tpt = 2, tile = 1024;
    bool tc_up = true;      // leaf P2M of the mixed Lagrange path on the tensor cores
    int shard = 0, nshards = 1;
    bool sym = true;        // symmetric near-field pairs once for both sides (bt_sym.cu)
};

// Autotuned shapes per device, kernel and approximation (bt_autotune,
// bt_tuning_set); process-wide.
std::mutex g_tune_mu;
bt_tuning g_tuned[16][16][3];
bool g_has_tuned[16][16][3];

bool tune_key_ok(int device, int kernel, int approx)
{
    return device >= 0 && device < 16 && kernel >= 0 && kernel < 16 && approx >= 0 && approx < 3;
}

EvalConfig tuned_shape(int device, int kernel, int approx)
{
    EvalConfig sh;
    if (!tune_key_ok(device, kernel, approx)) return sh;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_has_tuned[device][kernel][approx]) {
        const bt_tuning &t = g_tuned[device][kernel][approx];
        sh.queue = t.dispatch == BT_DISPATCH_QUEUE;
        sh.tpt = t.targets_per_thread;
        sh.tile = t.source_tile;
    }
    return sh;
}

int get_ctx(int device, DeviceCtx **out)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_err("no CUDA device available");
        return BT_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev || device >= 16) {
        set_err("invalid device ordinal %d", device);
        return BT_ERR_PARAM;
    }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    DeviceCtx &c = g_ctx[device];
    if (cudaSetDevice(device) != cudaSuccess) { set_err("cudaSetDevice failed"); return BT_ERR_CUDA; }
    // an error left by the caller's earlier work is not this call's
    cudaGetLastError();
    if (c.device < 0) {
        if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) {
            set_err("stream creation failed");
            return BT_ERR_CUDA;
        }
        for (auto &e : c.ev) cudaEventCreate(&e);
        if (cudaStreamCreateWithFlags(&c.fk.side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&c.fk.side2, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&c.fk.fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&c.fk.join, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&c.fk.join2, cudaEventDisableTiming) != cudaSuccess) {
            set_err("stream creation failed");
            return BT_ERR_CUDA;
        }
        c.device = device;
    }
    *out = &c;
    return BT_OK;
}

// Size accounting pass + allocation pass over the same sequence of requests.
struct Layout {
    std::vector<std::pair<void **, size_t>> reqs;
    template <typename T>
    void add(T **p, size_t count) { reqs.push_back({(void **)p, sizeof(T) * (count > 0 ? count : 1)}); }
    size_t total() const
    {
        size_t s = 0;
        for (auto &r : reqs) s = ((s + 255) & ~size_t(255)) + r.second;
        return s + 256;
    }
    void bind(Arena &a)
    {
        a.used = 0;
        for (auto &r : reqs) *r.first = a.take(r.second);
    }
};

#define CK(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            set_err("CUDA error %s at %s:%d", cudaGetErrorString(e_), __FILE__, __LINE__); \
            rc = BT_ERR_CUDA;                                                         \
            goto done;                                                                \
        }                                                                             \
    } while (0)

int validate(int nt, int ns, const void *tx, const void *ty, const void *tz, const void *sx, const void *sy,
             const void *sz, const void *sq, const void *out, const bt_params &p)
{
    if (nt < 0 || ns < 0) { set_err("negative particle count"); return BT_ERR_PARAM; }
    if ((nt > 0 && (!tx || !ty || !tz || !out)) || (ns > 0 && (!sx || !sy || !sz || !sq))) {
        // Particles_Validate (src/particles/particles.c:170-176) exits here
        set_err("one or more required particle arrays is unset");
        return BT_ERR_PARAM;
    }
    if (p.approx != LAGRANGE && p.approx != HERMITE) { set_err("invalid approximation %d", p.approx); return BT_ERR_PARAM; }
    if (p.sing != SKIPPING && p.sing != SUBTRACTION) {
        set_err("invalid singularity %d", p.sing);
        return BT_ERR_PARAM;
    }
    // kernels and the combinations the reference provides them in
    // (src/interaction_compute/interaction_compute_pc.c, _cp.c, _cc.c; the
    // others exit): Hermite for Coulomb, Yukawa, regularized Coulomb and
    // sin-over-r; grid outputs (CP, CC) for all but atan and MQ; subtraction
    // for Coulomb, Yukawa and the two regularized kernels in PC, and for
    // Coulomb and Yukawa with Lagrange in CP / CC
    // (interaction_compute_downpass.c:126-128)
    const int k = p.kernel;
    const bool known = k == COULOMB || k == YUKAWA || k == REGULARIZED_COULOMB || k == REGULARIZED_YUKAWA ||
                       k == ATAN || k == SIN_OVER_R || k == MQ || k == RBS_U || k == RBS_V || k == USER;
    if (!known) {
        set_err("kernel %d not provided", k);
        return BT_ERR_UNSUPPORTED;
    }
    const bool hermite_ok = k == COULOMB || k == YUKAWA || k == REGULARIZED_COULOMB || k == SIN_OVER_R;
    if (p.approx == HERMITE && !hermite_ok) {
        set_err("kernel %d has no Hermite form in the reference", k);
        return BT_ERR_UNSUPPORTED;
    }
    if ((k == ATAN || k == MQ) && p.ctype != PARTICLE_CLUSTER) {
        set_err("the atan and MQ kernels are provided for particle-cluster only, as in the reference");
        return BT_ERR_UNSUPPORTED;
    }
    if (p.sing == SUBTRACTION) {
        const bool ss_pc = k == COULOMB || k == YUKAWA || k == REGULARIZED_COULOMB ||
                           (k == REGULARIZED_YUKAWA && p.approx == LAGRANGE);
        const bool ss_grid = (k == COULOMB || k == YUKAWA) && p.approx == LAGRANGE;
        if (!(p.ctype == PARTICLE_CLUSTER ? ss_pc : ss_grid)) {
            set_err("singularity subtraction is not provided for kernel %d with this approximation and compute "
                    "type (the reference exits there)", k);
            return BT_ERR_UNSUPPORTED;
        }
    }
    if ((k == REGULARIZED_YUKAWA || k == ATAN || k == MQ || (k == REGULARIZED_COULOMB && p.sing == SUBTRACTION)) &&
        p.nkp < 2) {
        set_err("kernel %d needs two kernel parameters", k);
        return BT_ERR_PARAM;
    }
    if (p.ctype != PARTICLE_CLUSTER && p.ctype != CLUSTER_PARTICLE && p.ctype != CLUSTER_CLUSTER) {
        set_err("invalid compute type %d", p.ctype);
        return BT_ERR_PARAM;
    }
    if (p.ctype == CLUSTER_CLUSTER && p.approx == HERMITE) {
        // src/interaction_compute/interaction_compute_cc.c:146-147
        set_err("cluster-cluster Hermite is inoperable in the reference and not provided");
        return BT_ERR_UNSUPPORTED;
    }
    if (p.degree < 1 || p.degree > 12) { set_err("interpolation degree %d outside 1..12", p.degree); return BT_ERR_UNSUPPORTED; }
    if (p.maxs < 1 || p.maxt < 1) { set_err("leaf sizes must be >= 1"); return BT_ERR_PARAM; }
    if (!(p.theta > 0.0)) { set_err("theta must be > 0"); return BT_ERR_PARAM; }
    return BT_OK;
}

void hermite_ww(int n, double *ww)
{
    // src/clusters/clusters.c:1289-1300
    for (int i = 0; i <= n; i++) {
        double xx = i * M_PI / n;
        ww[i] = -cos(xx) / (2 * sin(xx) * sin(xx));
    }
    ww[0] = 0.25 * (n * n / 3.0 + 1.0 / 6.0);
    ww[n] = -ww[0];
}

// Chebyshev grids of every node: x0 + (cos(i pi / n) + 1) / 2 (x1 - x0) per
// axis, the same operations as bt_cheb_nodes (src/clusters/clusters.c:857-862)
// with the n+1 factors (cos + 1) / 2 computed once per call.
void fill_grids(const bt_tree &t, int n, hvec<double> &grid, hvec<double> &len)
{
    const int np1 = n + 1;
    double h[BT_MAX_DEGREE + 1];
    for (int i = 0; i <= n; i++) h[i] = (cos(i * M_PI / n) + 1.0) / 2.0;
    grid.resize((size_t)t.n * 3 * np1);
    len.resize((size_t)t.n * 3);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < t.n; i++) {
        double *g = grid.data() + (size_t)i * 3 * np1;
        const double lo[3] = {t.x0[i], t.y0[i], t.z0[i]}, hi[3] = {t.x1[i], t.y1[i], t.z1[i]};
        for (int a = 0; a < 3; a++) {
            for (int k = 0; k <= n; k++) g[a * np1 + k] = lo[a] + h[k] * (hi[a] - lo[a]);
            len[3 * (size_t)i + a] = hi[a] - lo[a];
        }
    }
}

// Work items (unit, chunk) sorted by decreasing cost so the block scheduler
// starts the longest work first.
std::vector<int2> make_items(int units, const int *count_of_unit, int chunk, const std::vector<double> &cost)
{
    // the items of a unit share its cost: a stable sort of the units, each
    // then expanded into its chunks in order, is the stable sort of the items
    std::vector<int> ord;
    size_t n = 0;
    for (int u = 0; u < units; u++)
        if (count_of_unit[u] > 0) {
            ord.push_back(u);
            n += (size_t)((count_of_unit[u] + chunk - 1) / chunk);
        }
    std::stable_sort(ord.begin(), ord.end(), [&cost](int a, int b) { return cost[a] > cost[b]; });
    std::vector<int2> out;
    out.reserve(n);
    for (int u : ord)
        for (int c = 0; c < (count_of_unit[u] + chunk - 1) / chunk; c++) out.push_back(make_int2(u, c));
    return out;
}

// Algorithmic FLOPs per pointwise interaction (FMA = 2): Coulomb 10
// (3 sub, 5 for r^2, 2 for the charge multiply-add; the reciprocal square
// root is a special-function op and not counted), regularized Coulomb 11,
// Yukawa 13 (+ kappa*r and the exp multiply); Hermite PC/CP 30.
double flops_per_eval(const bt_params &o, bool approx_side)
{
    if (approx_side && o.approx == HERMITE) return 30.0;
    return o.kernel == COULOMB ? 10.0 : o.kernel == YUKAWA ? 13.0 : 11.0;
}

void count_interactions(const bt_plan &pl, bt_report *r)
{
    // pointwise counts as src/drivers/treedriver.c:185-202, 467-483, 757-793
    const bt_params &o = pl.prm;
    long long P = o.P;
    r->num_pp = r->num_pc = r->num_cp = r->num_cc = 0;
    r->pp_ptwise = r->pc_ptwise = r->cp_ptwise = r->cc_ptwise = 0;
    if (o.ctype == PARTICLE_CLUSTER || o.ctype == CLUSTER_PARTICLE) {
        const bt_tree &trav = o.ctype == PARTICLE_CLUSTER ? pl.st : pl.tt;
        const bt_tree &bat = o.ctype == PARTICLE_CLUSTER ? pl.tt : pl.st;
        long long pp = 0, pa = 0, npp = 0, na_all = 0;
#pragma omp parallel for schedule(static) reduction(+ : pp, pa, npp, na_all)
        for (int i = 0; i < bat.nleaves; i++) {
            long long m = bat.numpar[bat.leaves[i]];
            for (int64_t k = pl.pp.off[i]; k < pl.pp.off[i + 1]; k++) pp += m * trav.numpar[pl.pp.idx[k]];
            long long na = pl.ap.off[i + 1] - pl.ap.off[i];
            pa += na * m * P;
            npp += pl.pp.off[i + 1] - pl.pp.off[i];
            na_all += na;
        }
        r->pp_ptwise = pp;
        r->num_pp = npp;
        if (o.ctype == PARTICLE_CLUSTER) { r->pc_ptwise = pa; r->num_pc = na_all; }
        else { r->cp_ptwise = pa; r->num_cp = na_all; }
    } else {
        for (int i = 0; i < pl.tt.n; i++) {
            long long m = pl.tt.numpar[i];
            for (int64_t k = pl.pp.off[i]; k < pl.pp.off[i + 1]; k++) r->pp_ptwise += m * pl.st.numpar[pl.pp.idx[k]];
            for (int64_t k = pl.cp.off[i]; k < pl.cp.off[i + 1]; k++) r->cp_ptwise += P * pl.st.numpar[pl.cp.idx[k]];
            r->pc_ptwise += (pl.pc.off[i + 1] - pl.pc.off[i]) * m * P;
            r->cc_ptwise += (pl.ap.off[i + 1] - pl.ap.off[i]) * P * P;
            r->num_pp += pl.pp.off[i + 1] - pl.pp.off[i];
            r->num_pc += pl.pc.off[i + 1] - pl.pc.off[i];
            r->num_cp += pl.cp.off[i + 1] - pl.cp.off[i];
            r->num_cc += pl.ap.off[i + 1] - pl.ap.off[i];
        }
    }
    // FLOPs of the particle-output evaluation kernel (PP + PC)
    long long pp = r->pp_ptwise, pc = (o.ctype == CLUSTER_PARTICLE) ? 0 : r->pc_ptwise;
    r->eval_flops = (long long)(pp * flops_per_eval(o, false) + pc * flops_per_eval(o, true));
}

// For every node: the range of its leaves in the tree's DFS leaf order (the
// leaves under a node are contiguous there because numbering is pre-order).
void leaf_ranges(const bt_tree &t, std::vector<int> &first, std::vector<int> &count)
{
    first.assign(t.n, 0);
    count.assign(t.n, 0);
    std::vector<int> pos(t.n, -1);
    for (int i = 0; i < t.nleaves; i++) pos[t.leaves[i]] = i;
    for (int v = t.n - 1; v >= 0; v--) {
        if (t.nchild[v] == 0) { first[v] = pos[v]; count[v] = 1; continue; }
        first[v] = first[t.child[8 * v]];
        int c = 0;
        for (int k = 0; k < t.nchild[v]; k++) c += count[t.child[8 * v + k]];
        count[v] = c;
    }
}

// Replace every node entry of a CSR by the leaves under it, in DFS order.
void expand_to_leaves(const bt_csr &in, const bt_tree &t, const std::vector<int> &first,
                      const std::vector<int> &count, std::vector<int64_t> &off, hvec<int> &idx)
{
    off.assign(in.rows + 1, 0);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < in.rows; r++) {
        int64_t c = 0;
        for (int64_t k = in.off[r]; k < in.off[r + 1]; k++) c += count[in.idx[k]];
        off[r + 1] = c;
    }
    for (int r = 0; r < in.rows; r++) off[r + 1] += off[r];
    idx.resize((size_t)off[in.rows]);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < in.rows; r++) {
        int64_t o = off[r];
        for (int64_t k = in.off[r]; k < in.off[r + 1]; k++) {
            const int s = in.idx[k];
            for (int l = 0; l < count[s]; l++) idx[o++] = t.leaves[first[s] + l];
        }
    }
}

// Build the host plan: copies, trees, lists.
// Systems of a call: nsys and the target / source offsets (a single system
// unless the call is batched).
struct Systems {
    int n = 1;
    std::vector<int64_t> toff, soff;
    Systems(int nt, int ns) : toff{0, nt}, soff{0, ns} {}
    Systems(int nsys, const long long *t, const long long *s) : n(nsys), toff(t, t + nsys + 1), soff(s, s + nsys + 1) {}
};

// Singularity subtraction inputs in caller order: target charges and
// source weights (host or device memory).
struct SsIn {
    const double *tq, *sw;
    bool on_device;
};

// Whether two host arrays hold the same bits (parallel compare).
bool same_host(const double *a, const double *b, size_t n)
{
    if (a == b) return true;
    const size_t CH = 1 << 16;
    const long nch = (long)((n + CH - 1) / CH);
    int diff = 0;
#pragma omp parallel for schedule(static) reduction(| : diff)
    for (long c = 0; c < nch; c++) {
        size_t b0 = (size_t)c * CH, len = std::min(CH, n - b0);
        diff |= memcmp(a + b0, b + b0, sizeof(double) * len) != 0;
    }
    return !diff;
}

// Build the host plan: copies, trees, lists.
void build_plan(bt_plan &pl, const Systems &sys, const double *tx, const double *ty, const double *tz,
                const double *sx, const double *sy, const double *sz, const double *sq)
{
    const int nt = (int)sys.toff[sys.n], ns = (int)sys.soff[sys.n];
    bt_parts_init(&pl.src, ns, sx, sy, sz, sq);
    bt_forest_build(&pl.st, &pl.src, sys.n, sys.soff.data(), pl.prm.maxs);
    // Targets at exactly the source positions with the same leaf size give
    // the same node sets (the build depends only on coordinates and leaf
    // size), so the target tree and permutation are copies of the source's.
    bool same = sys.toff == sys.soff && pl.prm.maxs == pl.prm.maxt && same_host(tx, sx, (size_t)nt) &&
                same_host(ty, sy, (size_t)nt) && same_host(tz, sz, (size_t)nt);
    if (same && nt > 0) {
        bt_parts_init(&pl.tgt, nt, pl.src.x, pl.src.y, pl.src.z, nullptr);
        memcpy(pl.tgt.order, pl.src.order, sizeof(int) * (size_t)nt);
        bt_tree_copy(&pl.tt, &pl.st);
        pl.same_tree = 1;
    } else {
        bt_parts_init(&pl.tgt, nt, tx, ty, tz, nullptr);
        bt_forest_build(&pl.tt, &pl.tgt, sys.n, sys.toff.data(), pl.prm.maxt);
    }
    bt_plan_lists(&pl);
}

void build_plan(bt_plan &pl, int nt, int ns, const double *tx, const double *ty, const double *tz,
                const double *sx, const double *sy, const double *sz, const double *sq)
{
    build_plan(pl, Systems(nt, ns), tx, ty, tz, sx, sy, sz, sq);
}

// Particles in tree order, resident on the device (GPU tree build).
struct DevParts {
    const double *sx = nullptr, *sy = nullptr, *sz = nullptr, *sq = nullptr;
    const double *tx = nullptr, *ty = nullptr, *tz = nullptr;
    const int *order = nullptr;     // target permutation
    const int *sorder = nullptr;    // source permutation
};

// The plan with both trees built on the GPU: the same trees and particle
// order as build_plan, the sorted particles kept in `tarena`.
int build_plan_gpu(DeviceCtx *ctx, Arena &tarena, bt_plan &pl, const Systems &sys, const double *tx,
                   const double *ty, const double *tz, const double *sx, const double *sy, const double *sz,
                   const double *sq, bool inputs_on_device, DevParts &dp)
{
    cudaStream_t st = ctx->stream;
    PhaseTimer pt;
    const bt_params &o = pl.prm;
    const int nt = (int)sys.toff[sys.n], ns = (int)sys.soff[sys.n];
    long long launches = 0;
    bool same = sys.toff == sys.soff && o.maxs == o.maxt;
    // host arrays: the comparison runs on another host thread while the
    // source tree is built (its inputs go to the device meanwhile)
    std::future<bool> same_fut;
    if (same && !inputs_on_device)
        same_fut = std::async(std::launch::async, [=] {
            return same_host(tx, sx, (size_t)nt) && same_host(ty, sy, (size_t)nt) && same_host(tz, sz, (size_t)nt);
        });
    const bool check_on_device = same && inputs_on_device && !(tx == sx && ty == sy && tz == sz);
    double *d_sx, *d_sy, *d_sz, *d_sq, *d_tx = nullptr, *d_ty = nullptr, *d_tz = nullptr;
    int *d_sord, *d_tord = nullptr;
    unsigned long long *d_flag;
    unsigned char *d_work;
    const size_t wbytes = std::max(bt::gpu_tree_work_bytes(ns, o.maxs, true, sys.n),
                                   bt::gpu_tree_work_bytes(nt, o.maxt, false, sys.n));
    Layout L;
    L.add(&d_sx, ns); L.add(&d_sy, ns); L.add(&d_sz, ns); L.add(&d_sq, ns); L.add(&d_sord, ns);
    L.add(&d_tx, nt); L.add(&d_ty, nt); L.add(&d_tz, nt); L.add(&d_tord, nt);
    L.add(&d_flag, 1); L.add(&d_work, wbytes);
    if (!tarena.reserve(L.total())) {
        set_err("device allocation of %zu bytes for the tree build failed", L.total());
        return BT_ERR_CUDA;
    }
    L.bind(tarena);
    if (check_on_device) {
        bool ex = false, ey = false, ez = false;
        int e = bt::gpu_arrays_equal(tx, sx, (size_t)nt, d_flag, &ex, st);
        if (!e) e = bt::gpu_arrays_equal(ty, sy, (size_t)nt, d_flag, &ey, st);
        if (!e) e = bt::gpu_arrays_equal(tz, sz, (size_t)nt, d_flag, &ez, st);
        if (e) { set_err("CUDA error %s in the coordinate comparison", cudaGetErrorString((cudaError_t)e)); return BT_ERR_CUDA; }
        launches += 3;
        same = ex && ey && ez;
    }
    bt::GtArrays sa{d_sx, d_sy, d_sz, d_sq, d_sord};
    int e = bt::gpu_build_forest(sys.n, sys.soff.data(), sx, sy, sz, sq, o.maxs, sa, d_work, wbytes, &pl.st, st,
                                 &launches);
    const char *which = "source";
    pt.mark("setup: source tree (GPU)");
    if (same_fut.valid()) {
        same = same_fut.get();
        pt.mark("setup: compare target/source arrays");
    }
    if (!e && !same) {
        bt::GtArrays ta{d_tx, d_ty, d_tz, nullptr, d_tord};
        which = "target";
        e = bt::gpu_build_forest(sys.n, sys.toff.data(), tx, ty, tz, nullptr, o.maxt, ta, d_work, wbytes, &pl.tt, st,
                                 &launches);
    }
    g_launches += launches;
    if (e) {
        set_err("CUDA error %s in the %s tree build (bt_gputree.cu:%d)", cudaGetErrorString((cudaError_t)e), which,
                bt::gpu_tree_fail_line());
        return BT_ERR_CUDA;
    }
    pl.src.n = ns;
    pl.tgt.n = nt;
    dp.sx = d_sx; dp.sy = d_sy; dp.sz = d_sz; dp.sq = d_sq; dp.sorder = d_sord;
    if (same) {
        bt_tree_copy(&pl.tt, &pl.st);
        pl.same_tree = 1;
        dp.tx = d_sx; dp.ty = d_sy; dp.tz = d_sz; dp.order = d_sord;
    } else {
        dp.tx = d_tx; dp.ty = d_ty; dp.tz = d_tz; dp.order = d_tord;
    }
    pt.mark("setup: target tree");
    // particle-cluster and cluster-particle lists: traversed on the GPU in the
    // tree build's work memory (free again now); cluster-cluster's dual
    // traversal, and a traversal that does not fit, run on the host
    int lrc = -1;
    if ((o.ctype == PARTICLE_CLUSTER || o.ctype == CLUSTER_PARTICLE) && !getenv("BARYTREE_B200_HOST_LISTS")) {
        const bt_tree *trav = o.ctype == PARTICLE_CLUSTER ? &pl.st : &pl.tt;
        const bt_tree *bat = o.ctype == PARTICLE_CLUSTER ? &pl.tt : &pl.st;
        long long gl = 0;
        lrc = bt::gpu_pc_lists(trav, bat, &o, d_work, wbytes, &pl.ap, &pl.pp, st, &gl);
        g_launches += gl;
        if (lrc > 0) {
            set_err("CUDA error %s in the interaction-list traversal", cudaGetErrorString((cudaError_t)lrc));
            return BT_ERR_CUDA;
        }
    }
    if (lrc == 0) {
        bt_csr_empty(&pl.pc, pl.ap.rows);
        bt_csr_empty(&pl.cp, pl.ap.rows);
        bt_plan_work_lists(&pl);
        pt.mark("setup: interaction lists (GPU traversal)");
    } else {
        bt_plan_lists(&pl);
        pt.mark("setup: interaction lists (host)");
    }
    return BT_OK;
}

// Everything the device sequence of one evaluation needs: the device arrays
// of a prepared plan and the few host-side sizes that shape the launches.
struct DevPlan {
    bool mixed = false, herm = false, need_src_clusters = false, need_tgt_grids = false;
    bool queue = false;     // mixed kernels on a device work queue
    int tpt = 2, tile = 1024;   // tile shape of the mixed particle-output kernel
    int fp64_tb = 1;            // targets per thread of the FP64 particle-output kernel
    bool base_full = true;      // proxies at the base degree for every node (else only the selected
                                // degrees' marked subtrees, the base degree among them)
    bool tc_up = false;         // leaf P2M on the tensor cores (bt_tc.cu)
    bool sharded = false;       // this call evaluates a share of the target leaves (others get 0)
    // symmetric near-field pairs (bt_sym.cu)
    int sym_npairs = 0;
    int sym_far_pairs = 0;      // the first pairs: boxes apart by more than the close-pair distance
    double *d_sbox = nullptr;   // node boxes (x0 x1 y0 y1 z0 z1) for the pairs within it
    int2 *d_sym_pairs = nullptr;
    int64_t *d_sym_slot = nullptr, *d_sym_in_off = nullptr, *d_sym_in_slot = nullptr;
    float *d_sym_partial = nullptr;
    int *d_err = nullptr;       // set by a tensor-core kernel whose bounded wait expired
    int n = 0, P = 0, ns = 0, nt = 0, max_np1 = 0, kernel = 0;
    double kp = 0.0;
    int S_n = 0, S_nleaves = 0, S_max_depth = 0, T_n = 0, T_nleaves = 0, T_max_depth = 0;
    std::vector<int> S_lvl_off, T_lvl_off, xdeg;
    int n_grid_items = 0, n_ev_items = 0, n_l2p_items = 0;
    double *d_sx = nullptr, *d_sy = nullptr, *d_sz = nullptr, *d_sq = nullptr, *d_tx = nullptr, *d_ty = nullptr, *d_tz = nullptr, *d_pot = nullptr, *d_sgrid = nullptr, *d_tgrid = nullptr, *d_slen = nullptr, *d_tlen = nullptr, *d_ww = nullptr, *d_Q = nullptr, *d_Phi = nullptr, *d_srad = nullptr, *d_trad = nullptr, *d_sctr = nullptr, *d_tctr = nullptr;
    int *d_sibeg = nullptr, *d_snum = nullptr, *d_snch = nullptr, *d_sch = nullptr, *d_sleaves = nullptr, *d_slvl = nullptr, *d_tibeg = nullptr, *d_tnum = nullptr, *d_tnch = nullptr, *d_tch = nullptr, *d_tpar = nullptr, *d_tleaves = nullptr, *d_tlvl = nullptr, *d_aidx = nullptr, *d_didx = nullptr, *d_ccidx = nullptr, *d_cpidx = nullptr, *d_order = nullptr, *d_queue = nullptr, *d_mxdidx = nullptr, *d_mxcpidx = nullptr;
    int64_t *d_aoff = nullptr, *d_doff = nullptr, *d_ccoff = nullptr, *d_cpoff = nullptr, *d_mxdoff = nullptr, *d_mxcpoff = nullptr;
    int2 *d_evitems = nullptr, *d_griditems = nullptr, *d_l2pitems = nullptr;
    float4 *d_spos = nullptr, *d_tpos = nullptr;
    float *d_Q32 = nullptr;
    unsigned char *d_mxdflag = nullptr, *d_adeg = nullptr;
    double *d_xgrid[BT_MAX_DEGREE + 1] = {}, *d_xQ[BT_MAX_DEGREE + 1] = {};
    float *d_xQ32[BT_MAX_DEGREE + 1] = {};
    // extra degree i: the leaves and per-level internal nodes that need its proxies
    int *d_xleaves[BT_MAX_DEGREE + 1] = {}, *d_xlvl[BT_MAX_DEGREE + 1] = {};
    std::vector<int> xleaf_n;
    std::vector<std::vector<int>> xlvl_off;
    double *d_out = nullptr;    // potentials in caller order (run_plan's own buffer)
    bool ss = false;                        // singularity subtraction
    double kp2 = 0.0, ss_c = 0.0;           // kernel_params[1]; correction constant
    double *d_tq = nullptr, *d_sw = nullptr, *d_qw = nullptr, *d_W = nullptr, *d_Phiw = nullptr;
    bt::HermChunk *d_hchunks = nullptr;     // Hermite P2M: particle chunks of every node
    int3 *d_hred = nullptr;                 // nodes with several chunks
    double *d_hpartial = nullptr;           // their partial moments
    int n_hchunks = 0, n_hred = 0;
};

// BT_ERR_TIMEOUT if a tensor-core kernel of the last evaluation gave up
// waiting for its MMAs (its flag is cleared at the start of every evaluation).
int check_device_error(const DevPlan &v, cudaStream_t st)
{
    if (!v.tc_up || !v.d_err) return BT_OK;
    int flag = 0;
    if (cudaMemcpyAsync(&flag, v.d_err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        set_err("reading the device error flag failed");
        return BT_ERR_CUDA;
    }
    if (flag) {
        set_err("a tensor-core wait expired in the upward pass");
        return BT_ERR_TIMEOUT;
    }
    return BT_OK;
}

// Arguments of the mixed particle-output kernel of a prepared plan.
bt::MixedTargetsArgs mixed_targets_args(const DevPlan &v)
{
    bt::MixedTargetsArgs a;
    memset(&a, 0, sizeof a);
    const int n = v.n;
    a.n = n; a.max_np1 = v.max_np1; a.nitems = v.n_ev_items; a.items = v.d_evitems; a.herm = v.herm;
    a.queue = v.queue ? v.d_queue + 1 : nullptr;
    a.tpt = v.tpt; a.tile = v.tile;
    a.leaf_node = v.d_tleaves; a.t_ibeg = v.d_tibeg; a.t_numpar = v.d_tnum; a.t_ctr = v.d_tctr; a.tpos = v.d_tpos;
    a.a_off = v.d_aoff; a.a_idx = v.d_aidx; a.a_deg = v.d_adeg;
    a.s_grid[n] = v.d_sgrid; a.Q32[n] = v.d_Q32;
    for (size_t i = 0; i < v.xdeg.size(); i++) { a.s_grid[v.xdeg[i]] = v.d_xgrid[i]; a.Q32[v.xdeg[i]] = v.d_xQ32[i]; }
    a.d_off = v.d_mxdoff; a.d_idx = v.d_mxdidx; a.d_flag = v.d_mxdflag; a.s_ibeg = v.d_sibeg; a.s_numpar = v.d_snum;
    a.s_ctr = v.d_sctr;
    a.spos = v.d_spos; a.kc = bt::mixed_kernel_constant(v.kernel, v.kp); a.pot = v.d_pot;
    a.t_rad = v.d_trad; a.s_rad = v.d_srad;
    a.tx64 = v.d_tx; a.ty64 = v.d_ty; a.tz64 = v.d_tz; a.sx64 = v.d_sx; a.sy64 = v.d_sy; a.sz64 = v.d_sz; a.sq64 = v.d_sq;
    a.kp = v.kp;
    return a;
}

// The device sequence of one evaluation (stream-ordered, no host
// synchronisation, so it can be captured into a CUDA graph): relative
// positions, upward pass, grid-output and particle-output kernels, downward
// pass, and the scatter of the potentials into caller order at scatter_out.
// ev: 5 events bracketing the phases, or nullptr.
int issue_plan(const DevPlan &v, cudaStream_t st, cudaEvent_t *ev, double *scatter_out, long long &launches,
               bool capturing = false, const Fork *fk = nullptr)
{
    // inside a stream capture an event becomes a record node of the graph
    // only when recorded as external
    auto record = [&](int k) {
        return capturing ? cudaEventRecordWithFlags(ev[k], st, cudaEventRecordExternal) : cudaEventRecord(ev[k], st);
    };
    int rc = BT_OK;
    const bool mixed = v.mixed, herm = v.herm, need_src_clusters = v.need_src_clusters, need_tgt_grids = v.need_tgt_grids;
    const int n = v.n, P = v.P, ns = v.ns, nt = v.nt;
    const std::vector<int> &xdeg = v.xdeg;
    auto d_sx = v.d_sx;
    auto d_sy = v.d_sy;
    auto d_sz = v.d_sz;
    auto d_sq = v.d_sq;
    auto d_tx = v.d_tx;
    auto d_ty = v.d_ty;
    auto d_tz = v.d_tz;
    auto d_pot = v.d_pot;
    auto d_sgrid = v.d_sgrid;
    auto d_tgrid = v.d_tgrid;
    auto d_slen = v.d_slen;
    auto d_tlen = v.d_tlen;
    auto d_ww = v.d_ww;
    auto d_Q = v.d_Q;
    auto d_Phi = v.d_Phi;
    auto d_sctr = v.d_sctr;
    auto d_tctr = v.d_tctr;
    auto d_sibeg = v.d_sibeg;
    auto d_snum = v.d_snum;
    auto d_snch = v.d_snch;
    auto d_sch = v.d_sch;
    auto d_sleaves = v.d_sleaves;
    auto d_slvl = v.d_slvl;
    auto d_tibeg = v.d_tibeg;
    auto d_tnum = v.d_tnum;
    auto d_tnch = v.d_tnch;
    auto d_tch = v.d_tch;
    auto d_tpar = v.d_tpar;
    auto d_tleaves = v.d_tleaves;
    auto d_tlvl = v.d_tlvl;
    auto d_aidx = v.d_aidx;
    auto d_didx = v.d_didx;
    auto d_ccidx = v.d_ccidx;
    auto d_cpidx = v.d_cpidx;
    auto d_order = v.d_order;
    auto d_queue = v.d_queue;
    auto d_mxcpidx = v.d_mxcpidx;
    auto d_aoff = v.d_aoff;
    auto d_doff = v.d_doff;
    auto d_ccoff = v.d_ccoff;
    auto d_cpoff = v.d_cpoff;
    auto d_mxcpoff = v.d_mxcpoff;
    auto d_evitems = v.d_evitems;
    auto d_griditems = v.d_griditems;
    auto d_l2pitems = v.d_l2pitems;
    auto d_spos = v.d_spos;
    auto d_tpos = v.d_tpos;
    auto d_Q32 = v.d_Q32;
    auto &d_xgrid = v.d_xgrid;
    auto &d_xQ = v.d_xQ;
    auto &d_xQ32 = v.d_xQ32;
    if (mixed) {
        bt::launch_rel_positions(v.S_nleaves, d_sleaves, d_sibeg, d_snum, d_sctr, d_sx, d_sy, d_sz, d_sq, d_spos, st);
        bt::launch_rel_positions(v.T_nleaves, d_tleaves, d_tibeg, d_tnum, d_tctr, d_tx, d_ty, d_tz, nullptr, d_tpos, st);
        launches += 2;
    }
    if (ev) CK(record(0));
    // upward pass
    if (v.tc_up) CK(cudaMemsetAsync(v.d_err, 0, sizeof(int), st));
    if (need_src_clusters && ns > 0 && v.ss) {
        // subtraction: proxies of q*w (Q) and of w (W) by the same passes
        const double *charges[2] = {v.d_qw, v.d_sw};
        double *proxies[2] = {d_Q, v.d_W};
        for (int k = 0; k < 2; k++) {
            if (herm) {
                bt::launch_p2m_hermite(n, v.n_hchunks, v.d_hchunks, v.n_hred, v.d_hred, d_sgrid, d_slen, d_ww, d_sx,
                                       d_sy, d_sz, charges[k], proxies[k], v.d_hpartial, st);
                launches += v.n_hred > 0 ? 2 : 1;
                continue;
            }
            bt::launch_p2m(n, false, v.S_nleaves, d_sleaves, v.S_n, d_sibeg, d_snum, d_sgrid, d_slen, d_ww, d_sx, d_sy,
                           d_sz, charges[k], proxies[k], st);
            launches++;
            for (int l = v.S_max_depth - 1; l >= 0; l--) {
                int cnt = v.S_lvl_off[l + 1] - v.S_lvl_off[l];
                if (cnt > 0) {
                    bt::launch_m2m(n, cnt, d_slvl + v.S_lvl_off[l], d_snch, d_sch, d_sgrid, proxies[k], st);
                    launches++;
                }
            }
        }
    } else if (need_src_clusters && ns > 0) {
        // the base degree at every node, unless a learned selection lists it
        // among its degrees (computed below under the nodes that use it)
        if (v.base_full) {
            static_assert(sizeof(bt::HermChunkTc) == sizeof(bt::HermChunk), "the two chunk types share one array");
            if (herm && v.tc_up && bt::p2m_hermite_tc_supported(n)) {
                // mixed Hermite: the 8 moments per chunk on the tensor cores, then
                // the same reduction of the nodes with several chunks
                bt::launch_p2m_hermite_tc(n, v.n_hchunks, reinterpret_cast<const bt::HermChunkTc *>(v.d_hchunks), d_sgrid,
                                          d_slen, d_ww, d_sx, d_sy, d_sz, d_sq, d_Q, v.d_hpartial, v.d_err, st);
                bt::launch_hermite_reduce(n, v.n_hred, v.d_hred, v.d_hpartial, d_Q, st);
                launches += v.n_hred > 0 ? 2 : 1;
            } else if (herm) {
                bt::launch_p2m_hermite(n, v.n_hchunks, v.d_hchunks, v.n_hred, v.d_hred, d_sgrid, d_slen, d_ww, d_sx, d_sy,
                                       d_sz, d_sq, d_Q, v.d_hpartial, st);
                launches += v.n_hred > 0 ? 2 : 1;
            } else if (v.tc_up && bt::p2m_tc_supported(n)) {
                bt::launch_p2m_tc(n, v.S_nleaves, d_sleaves, d_sibeg, d_snum, d_sgrid, d_sx, d_sy, d_sz, d_sq, d_Q, v.d_err,
                                  st);
                launches++;
            } else {
                bt::launch_p2m(n, false, v.S_nleaves, d_sleaves, v.S_n, d_sibeg, d_snum, d_sgrid, d_slen, d_ww, d_sx, d_sy,
                               d_sz, d_sq, d_Q, st);
                launches++;
            }
            if (!herm) {
                for (int l = v.S_max_depth - 1; l >= 0; l--) {
                    int cnt = v.S_lvl_off[l + 1] - v.S_lvl_off[l];
                    if (cnt > 0) {
                        bt::launch_m2m(n, cnt, d_slvl + v.S_lvl_off[l], d_snch, d_sch, d_sgrid, d_Q, st);
                        launches++;
                    }
                }
            }
            if (mixed) {
                bt::launch_to_f32((size_t)v.S_n * P * (herm ? 8 : 1), d_Q, d_Q32, st);
                launches++;
            }
        }
        // proxy charges at the degrees chosen per interaction: independent
        // chains (P2M, M2M level by level, FP32 copy), spread over the main
        // stream and the two side streams so that one degree's small
        // upper-level launches overlap another's
        const bool xfork = xdeg.size() > 1 && fk && fk->side && fk->side2;
        cudaStream_t xst[3] = {st, st, st};
        if (xfork) {
            CK(cudaEventRecord(fk->fork, st));
            CK(cudaStreamWaitEvent(fk->side, fk->fork, 0));
            CK(cudaStreamWaitEvent(fk->side2, fk->fork, 0));
            xst[1] = fk->side;
            xst[2] = fk->side2;
        }
        for (size_t i = 0; i < xdeg.size(); i++) {
            const int d = xdeg[i];
            const int nl = v.xleaf_n[i];
            cudaStream_t ds = xst[i % 3];
            if (nl > 0) {
                if (v.tc_up && bt::p2m_tc_supported(d))
                    bt::launch_p2m_tc(d, nl, v.d_xleaves[i], d_sibeg, d_snum, d_xgrid[i], d_sx, d_sy, d_sz, d_sq,
                                      d_xQ[i], v.d_err, ds);
                else
                    bt::launch_p2m(d, false, nl, v.d_xleaves[i], v.S_n, d_sibeg, d_snum, d_xgrid[i], d_slen, d_ww,
                                   d_sx, d_sy, d_sz, d_sq, d_xQ[i], ds);
                launches++;
            }
            const std::vector<int> &lo = v.xlvl_off[i];
            for (int l = v.S_max_depth - 1; l >= 0; l--) {
                int cnt = lo[l + 1] - lo[l];
                if (cnt > 0) {
                    bt::launch_m2m(d, cnt, v.d_xlvl[i] + lo[l], d_snch, d_sch, d_xgrid[i], d_xQ[i], ds);
                    launches++;
                }
            }
            bt::launch_to_f32((size_t)v.S_n * (d + 1) * (d + 1) * (d + 1), d_xQ[i], d_xQ32[i], ds);
            launches++;
        }
        if (xfork) {
            CK(cudaGetLastError());
            CK(cudaEventRecord(fk->join, fk->side));
            CK(cudaEventRecord(fk->join2, fk->side2));
            CK(cudaStreamWaitEvent(st, fk->join, 0));
            CK(cudaStreamWaitEvent(st, fk->join2, 0));
        }
    }
    CK(cudaGetLastError());
    if (ev) CK(record(1));
    // grid-output evaluation (CP, M2L) and L2L
    if (mixed && v.queue) CK(cudaMemsetAsync(d_queue, 0, 2 * sizeof(int), st));
    // a shard evaluates the grids of its own nodes only; the others start at 0
    if (need_tgt_grids && nt > 0 && v.sharded) {
        CK(cudaMemsetAsync(d_Phi, 0, sizeof(double) * (size_t)v.T_n * P * (herm ? 8 : 1), st));
        if (v.ss) CK(cudaMemsetAsync(v.d_Phiw, 0, sizeof(double) * (size_t)v.T_n * P, st));
    }
    if (need_tgt_grids && nt > 0 && v.ss) {
        bt::SsGridsArgs g;
        g.n = n; g.nitems = v.n_grid_items; g.items = d_griditems; g.t_grid = d_tgrid;
        g.c_off = d_ccoff; g.c_idx = d_ccidx; g.p_off = d_cpoff; g.p_idx = d_cpidx;
        g.s_ibeg = d_sibeg; g.s_numpar = d_snum; g.s_grid = d_sgrid; g.Q = d_Q; g.W = v.d_W;
        g.sx = d_sx; g.sy = d_sy; g.sz = d_sz; g.sq = d_sq; g.sw = v.d_sw; g.kp = v.kp;
        g.Phi_q = d_Phi; g.Phi_w = v.d_Phiw;
        bt::launch_ss_grids(v.kernel, g, st);
        launches++;
    } else if (need_tgt_grids && nt > 0 && mixed) {
        bt::MixedGridsArgs g;
        g.n = n; g.nitems = v.n_grid_items; g.items = d_griditems; g.t_grid = d_tgrid; g.t_ctr = d_tctr;
        g.queue = v.queue ? d_queue : nullptr;
        g.c_off = d_ccoff; g.c_idx = d_ccidx; g.p_off = d_mxcpoff; g.p_idx = d_mxcpidx;
        g.s_ibeg = d_sibeg; g.s_numpar = d_snum; g.s_grid = d_sgrid; g.s_ctr = d_sctr; g.Q32 = d_Q32;
        g.spos = d_spos; g.kc = bt::mixed_kernel_constant(v.kernel, v.kp); g.Phi = d_Phi;
        bt::launch_eval_grids_mixed(v.kernel, g, st);
        launches++;
    } else if (need_tgt_grids && nt > 0) {
        bt::EvalGridsArgs g;
        g.n = n; g.nitems = v.n_grid_items; g.items = d_griditems; g.t_grid = d_tgrid;
        g.c_off = d_ccoff; g.c_idx = d_ccidx; g.p_off = d_cpoff; g.p_idx = d_cpidx;
        g.s_ibeg = d_sibeg; g.s_numpar = d_snum; g.s_grid = d_sgrid; g.Q = d_Q;
        g.sx = d_sx; g.sy = d_sy; g.sz = d_sz; g.sq = d_sq; g.kp = v.kp; g.kp2 = v.kp2; g.Phi = d_Phi;
        bt::launch_eval_grids(v.kernel, herm, g, st);
        launches++;
    }
    CK(cudaGetLastError());
    if (ev) CK(record(2));
    // particle-output evaluation (PC, PP); a shard leaves the other targets at 0
    if (nt > 0 && v.sharded) CK(cudaMemsetAsync(d_pot, 0, sizeof(double) * (size_t)nt, st));
    if (nt > 0 && v.ss) {
        bt::SsTargetsArgs a;
        a.n = n; a.nitems = v.n_ev_items; a.items = d_evitems; a.leaf_node = d_tleaves;
        a.t_ibeg = d_tibeg; a.t_numpar = d_tnum; a.a_off = d_aoff; a.a_idx = d_aidx; a.d_off = d_doff; a.d_idx = d_didx;
        a.s_ibeg = d_sibeg; a.s_numpar = d_snum; a.s_grid = d_sgrid; a.Q = d_Q; a.W = v.d_W;
        a.sx = d_sx; a.sy = d_sy; a.sz = d_sz; a.sq = d_sq; a.sw = v.d_sw;
        a.tx = d_tx; a.ty = d_ty; a.tz = d_tz; a.tq = v.d_tq; a.kp = v.kp; a.kp2 = v.kp2; a.pot = d_pot;
        bt::launch_ss_targets(v.kernel, herm, a, st);
        launches++;
    } else if (nt > 0 && mixed) {
        const bt::MixedTargetsArgs a = mixed_targets_args(v);
        // the symmetric pairs write only their own partial sums: their two
        // kernels run beside the particle-output kernel on two more streams,
        // joined before the gather adds them into the potentials
        const bool fork = v.sym_npairs > 0 && fk && fk->side && fk->side2;
        cudaStream_t sst = st, sst2 = st;
        if (fork) {
            CK(cudaEventRecord(fk->fork, st));
            CK(cudaStreamWaitEvent(fk->side, fk->fork, 0));
            CK(cudaStreamWaitEvent(fk->side2, fk->fork, 0));
            sst = fk->side;
            sst2 = fk->side2;
        }
        if (v.sym_npairs > 0) {
            bt::SymArgs y;
            y.npairs = v.sym_npairs; y.pair = v.d_sym_pairs; y.slot = v.d_sym_slot;
            y.ibeg = v.d_sibeg; y.numpar = v.d_snum; y.ctr = v.d_sctr; y.pos = v.d_spos;
            y.partial = v.d_sym_partial; y.kc = (float)bt::mixed_kernel_constant(v.kernel, v.kp);
            y.rad = v.d_srad; y.box = v.d_sbox; y.x64 = v.d_sx; y.y64 = v.d_sy; y.z64 = v.d_sz; y.q64 = v.d_sq;
            y.kp = v.kp;
            bt::SymArgs yc = y;
            y.npairs = v.sym_far_pairs;
            yc.npairs = v.sym_npairs - v.sym_far_pairs;
            yc.pair += v.sym_far_pairs;
            yc.slot += v.sym_far_pairs;
            bt::launch_pp_sym(v.kernel, y, sst);
            bt::launch_pp_sym_close(v.kernel, yc, sst2);
            launches += (y.npairs > 0) + (yc.npairs > 0);
        }
        bt::launch_eval_targets_mixed(v.kernel, a, st);
        launches++;
        if (fork) {
            CK(cudaGetLastError());
            CK(cudaEventRecord(fk->join, sst));
            CK(cudaEventRecord(fk->join2, sst2));
            CK(cudaStreamWaitEvent(st, fk->join, 0));
            CK(cudaStreamWaitEvent(st, fk->join2, 0));
        }
        if (v.sym_npairs > 0) {
            bt::SymGatherArgs g;
            g.nleaves = v.T_nleaves; g.leaf_node = v.d_tleaves; g.ibeg = v.d_sibeg; g.numpar = v.d_snum;
            g.in_off = v.d_sym_in_off; g.in_slot = v.d_sym_in_slot; g.partial = v.d_sym_partial; g.pot = d_pot;
            bt::launch_sym_gather(g, st);
            launches++;
        }
    } else if (nt > 0) {
        bt::EvalTargetsArgs a;
        a.n = n; a.nitems = v.n_ev_items; a.items = d_evitems; a.leaf_node = d_tleaves;
        a.t_ibeg = d_tibeg; a.t_numpar = d_tnum; a.a_off = d_aoff; a.a_idx = d_aidx; a.d_off = d_doff; a.d_idx = d_didx;
        a.s_ibeg = d_sibeg; a.s_numpar = d_snum; a.s_grid = d_sgrid; a.Q = d_Q;
        a.sx = d_sx; a.sy = d_sy; a.sz = d_sz; a.sq = d_sq; a.tx = d_tx; a.ty = d_ty; a.tz = d_tz;
        a.kp = v.kp; a.kp2 = v.kp2; a.pot = d_pot; a.tb = v.fp64_tb;
        bt::launch_eval_targets(v.kernel, herm, a, st);
        launches++;
    }
    CK(cudaGetLastError());
    if (ev) CK(record(3));
    // downward pass
    if (need_tgt_grids && nt > 0) {
        if (!herm) {
            for (int l = 0; l < v.T_max_depth; l++) {
                int cnt = v.T_lvl_off[l + 1] - v.T_lvl_off[l];
                if (cnt > 0) {
                    bt::launch_l2l(n, cnt, d_tlvl + v.T_lvl_off[l], d_tnch, d_tch, d_tgrid, d_Phi, st);
                    launches++;
                }
            }
        }
        if (v.tc_up && !herm && !v.ss && bt::l2p_tc_supported(n))
            // mixed Lagrange: the leaf interpolation as a GEMM on the tensor cores
            bt::launch_l2p_tc(n, v.n_l2p_items, d_l2pitems, d_tleaves, d_tibeg, d_tnum, d_tgrid, d_Phi, d_tx, d_ty,
                              d_tz, d_pot, v.d_err, st);
        else
            bt::launch_l2p(n, herm, v.n_l2p_items, d_l2pitems, d_tleaves, d_tpar, d_tibeg, d_tnum, d_tgrid,
                           d_tlen, d_ww, d_Phi, d_tx, d_ty, d_tz, d_pot, st);
        launches++;
        if (v.ss) {
            // the weight field, interpolated and multiplied by -tq per target
            for (int l = 0; l < v.T_max_depth; l++) {
                int cnt = v.T_lvl_off[l + 1] - v.T_lvl_off[l];
                if (cnt > 0) {
                    bt::launch_l2l(n, cnt, d_tlvl + v.T_lvl_off[l], d_tnch, d_tch, d_tgrid, v.d_Phiw, st);
                    launches++;
                }
            }
            bt::launch_l2p(n, false, v.n_l2p_items, d_l2pitems, d_tleaves, d_tpar, d_tibeg, d_tnum, d_tgrid,
                           d_tlen, d_ww, v.d_Phiw, d_tx, d_ty, d_tz, d_pot, st, v.d_tq);
            launches++;
        }
    }
    if (v.ss && nt > 0) {
        // subtraction correction (InteractionCompute_SubtractionPotentialCorrection,
        // src/interaction_compute/interaction_compute_correction.c:22-45)
        // (a shard: the targets of its own leaves, through the work items)
        if (v.sharded)
            bt::launch_ss_correction_items(v.n_ev_items, d_evitems, bt::ss_chunk(), d_tleaves, d_tibeg, d_tnum, v.ss_c,
                                           v.d_tq, d_pot, st);
        else
            bt::launch_ss_correction(nt, v.ss_c, v.d_tq, d_pot, st);
        launches++;
    }
    CK(cudaGetLastError());
    if (ev) CK(record(4));
    bt::launch_scatter(nt, d_order, d_pot, scatter_out, st);
    launches++;
    CK(cudaGetLastError());
done:
    return rc;
}

// Device evaluation of a built plan; writes potentials in caller order to out_host.
// execute = false: prepare only (uploads done, the device sequence not
// issued), for capture into a graph by the caller.
int run_plan(DeviceCtx *ctx, Arena &arena, bt_plan &pl, double *out, bool out_on_device, bt_report *rep,
             const DevParts *dp = nullptr, const EvalConfig &shape = EvalConfig(), DevPlan *dv_out = nullptr, bool execute = true,
             const SsIn *ss = nullptr)
{
    const bt_params &o = pl.prm;
    const int n = o.degree, P = o.P;
    const bool herm = o.approx == HERMITE;
    const int nq = herm ? 8 : 1;
    const bt_tree &S = pl.st, &T = pl.tt;
    const int ns = pl.src.n, nt = pl.tgt.n;
    cudaStream_t st = ctx->stream;
    int rc = BT_OK;
    double t0 = now_ms();
    PhaseTimer pt;
    long long launches = 0;

    hvec<double> sgrid, slen, tgrid, tlen;
    fill_grids(S, n, sgrid, slen);
    fill_grids(T, n, tgrid, tlen);
    pt.mark("plan: grids at the base degree");
    // further degrees used by a learned per-interaction selection (mixed path)
    std::vector<int> xdeg;
    std::vector<hvec<double>> xgrid;
    int64_t n_approx = pl.t_approx.off[pl.t_approx.rows];
    if (pl.a_deg) {
        bool used[BT_MAX_DEGREE + 1] = {};
#pragma omp parallel
        {
            bool u[BT_MAX_DEGREE + 1] = {};
#pragma omp for schedule(static)
            for (int64_t k = 0; k < n_approx; k++) u[pl.a_deg[k]] = true;
#pragma omp critical
            for (int d = 0; d <= BT_MAX_DEGREE; d++) used[d] = used[d] || u[d];
        }
        // the base degree is one of them: a selection uses it only where it
        // chose it, so its proxies too are computed only under those nodes
        for (int d = 1; d <= BT_MAX_DEGREE; d++)
            if (used[d]) xdeg.push_back(d);
        xgrid.resize(xdeg.size());
        hvec<double> tmp;
        for (size_t i = 0; i < xdeg.size(); i++) fill_grids(S, xdeg[i], xgrid[i], tmp);
    }
    pt.mark("plan: grids at the selected degrees");
    // Each extra degree needs proxies only at the source nodes some
    // interaction uses it for: its P2M and M2M run over the leaves and
    // internal nodes under those nodes (pre-order numbering: a node's
    // children come after it, so one forward sweep marks the subtrees).
    std::vector<std::vector<int>> xleaves(xdeg.size()), xlvl(xdeg.size()), xlvl_off(xdeg.size());
    if (!xdeg.empty() && S.n > 0) {
        const size_t X = xdeg.size();
        int slot[BT_MAX_DEGREE + 1];
        for (int d = 0; d <= BT_MAX_DEGREE; d++) slot[d] = -1;
        for (size_t i = 0; i < X; i++) slot[xdeg[i]] = (int)i;
        std::vector<unsigned char> need((size_t)S.n * X, 0);
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < n_approx; k++) {
            const int sl = slot[pl.a_deg[k]];
            if (sl < 0) continue;
            // most entries find their node marked already: read first, so
            // the threads do not keep pulling the same cache lines for writes
            unsigned char *f = &need[(size_t)pl.t_approx.idx[k] * X + sl];
            if (!__atomic_load_n(f, __ATOMIC_RELAXED)) __atomic_store_n(f, (unsigned char)1, __ATOMIC_RELAXED);
        }
        for (int v = 0; v < S.n; v++)
            for (int c = 0; c < S.nchild[v]; c++) {
                const int ch = S.child[8 * (size_t)v + c];
                for (size_t i = 0; i < X; i++) need[(size_t)ch * X + i] |= need[(size_t)v * X + i];
            }
        for (size_t i = 0; i < X; i++) {
            for (int u = 0; u < S.nleaves; u++)
                if (need[(size_t)S.leaves[u] * X + i]) xleaves[i].push_back(S.leaves[u]);
            xlvl_off[i].assign(S.max_depth + 1, 0);
            for (int l = 0; l < S.max_depth; l++) {
                if (S.lvl_off)
                    for (int k = S.lvl_off[l]; k < S.lvl_off[l + 1]; k++)
                        if (need[(size_t)S.lvl_nodes[k] * X + i]) xlvl[i].push_back(S.lvl_nodes[k]);
                xlvl_off[i][l + 1] = (int)xlvl[i].size();
            }
        }
    }
    int max_np1 = n + 1;
    for (int d : xdeg) max_np1 = std::max(max_np1, d + 1);
    double ww[BT_MAX_DEGREE + 1];
    hermite_ww(n, ww);
    pt.mark("plan: Chebyshev grids");

    // work items
    const bool need_src_clusters = (o.ctype != CLUSTER_PARTICLE);
    const bool need_tgt_grids = (o.ctype != PARTICLE_CLUSTER);
    std::vector<int> leaf_count(T.nleaves);
    std::vector<double> leaf_cost(T.nleaves, 0.0);
#pragma omp parallel for schedule(static)
    for (int u = 0; u < T.nleaves; u++) {
        leaf_count[u] = T.numpar[T.leaves[u]];
        double c = 0;
        if (pl.a_deg) {
            for (int64_t k = pl.t_approx.off[u]; k < pl.t_approx.off[u + 1]; k++) {
                double d1 = pl.a_deg[k] + 1;
                c += d1 * d1 * d1;
            }
        } else {
            c += (double)(pl.t_approx.off[u + 1] - pl.t_approx.off[u]) * P * nq;
        }
        for (int64_t k = pl.t_direct.off[u]; k < pl.t_direct.off[u + 1]; k++) c += S.numpar[pl.t_direct.idx[k]];
        leaf_cost[u] = c;
    }
    const bool ssm = ss != nullptr;
    // mixed precision: Lagrange, and Hermite particle-cluster (its far field
    // in FP32 over the 8 moments); Hermite grid outputs and subtraction
    // evaluate in FP64
    const bool mixed = o.precision == BT_PRECISION_MIXED && !ssm && (!herm || o.ctype == PARTICLE_CLUSTER) &&
                       o.kernel <= REGULARIZED_COULOMB;
    // grid-output cost per target node (CP and CC): the work-item order of
    // the grid evaluation, and for a sharded call the share of the leaves
    // under the node
    std::vector<double> gcost;
    if (need_tgt_grids) {
        gcost.assign(T.n, 0.0);
        for (int i = 0; i < T.n; i++) {
            double c = (double)(pl.g_cc.off[i + 1] - pl.g_cc.off[i]) * P;
            for (int64_t k = pl.g_cp.off[i]; k < pl.g_cp.off[i + 1]; k++) c += S.numpar[pl.g_cp.idx[k]] * nq;
            gcost[i] = c;
        }
    }
    // target sharding: the nodes whose grid outputs this shard evaluates
    // (the owned leaves and their ancestors)
    std::vector<unsigned char> tnode_need;
    if (shape.nshards > 1) {
        // contiguous runs of target leaves (tree order) of about equal cost;
        // leaf u belongs to the shard that holds the middle of its cost
        // interval.  A node's grid outputs serve the leaves under it, so its
        // cost is spread over them by particle count.
        std::vector<double> scost(leaf_cost);
        if (need_tgt_grids)
            for (int u = 0; u < T.nleaves; u++) {
                const int leaf = T.leaves[u];
                for (int v = leaf; v >= 0; v = T.parent[v])
                    if (T.numpar[v] > 0) scost[u] += gcost[v] * T.numpar[leaf] / T.numpar[v];
            }
        double total = 0.0;
        for (int u = 0; u < T.nleaves; u++) total += scost[u];
        double before = 0.0;
        for (int u = 0; u < T.nleaves; u++) {
            const double mid = before + 0.5 * scost[u];
            before += scost[u];
            int k = total > 0 ? (int)(mid / total * shape.nshards) : u % shape.nshards;
            if (k >= shape.nshards) k = shape.nshards - 1;
            if (k != shape.shard) leaf_count[u] = 0;
        }
        if (need_tgt_grids) {
            tnode_need.assign(T.n, 0);
            for (int u = 0; u < T.nleaves; u++)
                if (leaf_count[u] > 0)
                    for (int v = T.leaves[u]; v >= 0 && !tnode_need[v]; v = T.parent[v]) tnode_need[v] = 1;
        }
    }
    // FP64 particle-output kernel: two targets per thread where the items fill the GPU
    const int fp64_tb = (!mixed && !ssm) ? bt::fp64_targets_per_thread(T.nleaves, leaf_count.data()) : 1;
    std::vector<int2> ev_items =
        make_items(T.nleaves, leaf_count.data(),
                   mixed ? bt::mixed_targets_chunk() : ssm ? bt::ss_chunk() : bt::fp64_targets_chunk(fp64_tb),
                   leaf_cost);
    std::vector<int2> grid_items, l2p_items;
    if (need_tgt_grids) {
        std::vector<int> pcount(T.n, P);
        if (!tnode_need.empty())
            for (int i = 0; i < T.n; i++) pcount[i] = tnode_need[i] ? P : 0;
        grid_items = make_items(T.n, pcount.data(), 128, gcost);
        std::vector<double> lcost(T.nleaves, 1.0);
        l2p_items = make_items(T.nleaves, leaf_count.data(), 128, lcost);
    }
    // mixed precision: Lagrange only (Hermite evaluates in FP64); node
    // centres, leaf-expanded near-field / CP lists, and per near-field entry
    // whether the two leaves' boxes lie within the close-pair distance (only
    // then can a pair be close, or a target coincide with a source)
    std::vector<double> sctr, tctr;
    std::vector<int64_t> mx_doff, mx_cpoff;
    hvec<int> mx_didx, mx_cpidx;
    hvec<unsigned char> mx_dflag;
    if (mixed) {
        sctr.resize(3 * (size_t)S.n);
        tctr.resize(3 * (size_t)T.n);
        for (int i = 0; i < S.n; i++) { sctr[3 * i] = S.xm[i]; sctr[3 * i + 1] = S.ym[i]; sctr[3 * i + 2] = S.zm[i]; }
        for (int i = 0; i < T.n; i++) { tctr[3 * i] = T.xm[i]; tctr[3 * i + 1] = T.ym[i]; tctr[3 * i + 2] = T.zm[i]; }
        std::vector<int> lf, lc;
        leaf_ranges(S, lf, lc);
        expand_to_leaves(pl.t_direct, S, lf, lc, mx_doff, mx_didx);
        expand_to_leaves(pl.g_cp, S, lf, lc, mx_cpoff, mx_cpidx);
        mx_dflag.resize(mx_didx.size());
#pragma omp parallel for schedule(static)
        for (int u = 0; u < T.nleaves; u++) {
            int t = T.leaves[u];
            for (int64_t k = mx_doff[u]; k < mx_doff[u + 1]; k++) {
                int s = mx_didx[k];
                double gx = std::max(0.0, std::max(S.x0[s] - T.x1[t], T.x0[t] - S.x1[s]));
                double gy = std::max(0.0, std::max(S.y0[s] - T.y1[t], T.y0[t] - S.y1[s]));
                double gz = std::max(0.0, std::max(S.z0[s] - T.z1[t], T.z0[t] - S.z1[s]));
                double rr = bt::MX_CLOSE_FRAC * (T.rad[t] + S.rad[s]);
                mx_dflag[k] = gx * gx + gy * gy + gz * gz <= 1.0625 * rr * rr ? 1 : 0;
            }
        }
    }
    pt.mark("plan: work items and near-field lists");
    // Symmetric near-field pairs: with the targets being the sources and a
    // symmetric kernel, leaf pairs {A, B} (A != B) that hold each other as
    // near-field entries are evaluated once for both sides (bt_sym.cu) and
    // leave the per-target lists.  Every pass runs per unit in parallel.  The
    // pairs whose boxes are farther apart than the close-pair distance come
    // first, then the pairs within it (their own kernel); each group is
    // numbered by head unit (A < B), then by partner node, so the numbering
    // does not depend on the thread count.
    hvec<int2> sym_pairs;
    hvec<int64_t> sym_slot, sym_in_slot;
    std::vector<int64_t> sym_in_off;
    int64_t sym_total = 0, sym_far_pairs = 0;
    int max_leaf = 0;
    for (int u = 0; u < T.nleaves; u++) max_leaf = std::max(max_leaf, T.numpar[T.leaves[u]]);
    if (mixed && pl.same_tree && shape.sym && max_leaf <= bt::SYM_MAX_LEAF &&
        (o.kernel == COULOMB || o.kernel == YUKAWA || o.kernel == REGULARIZED_COULOMB) && T.nleaves > 1) {
        const int NU = T.nleaves;
        std::vector<int> unit_of(T.n, -1);
        for (int u = 0; u < NU; u++) unit_of[T.leaves[u]] = u;
        // a pair belongs to the shard that owns its head (the lower leaf):
        // that shard evaluates it and gathers both sides, the partner's side
        // into targets another shard owns (the combining sum adds them)
        std::vector<unsigned char> owned(NU, 1);
        if (shape.nshards > 1)
            for (int u = 0; u < NU; u++) owned[u] = leaf_count[u] > 0;
        const int64_t ne = mx_doff[NU];
        // per unit: its partners (other leaves), sorted by node, each with the
        // list entry it came from and whether the boxes are within the
        // close-pair distance (the same test from both sides)
        hvec<int> far(ne), fent(ne);
        hvec<unsigned char> fnear(ne);
        std::vector<int64_t> far_end(NU);
#pragma omp parallel
        {
            std::vector<uint64_t> keys;
#pragma omp for schedule(static)
            for (int u = 0; u < NU; u++) {
                const int A = T.leaves[u];
                keys.clear();
                for (int64_t k = mx_doff[u]; k < mx_doff[u + 1]; k++) {
                    const int B = mx_didx[k];
                    if (B == A || unit_of[B] < 0) continue;
                    keys.push_back(((uint64_t)(uint32_t)B << 32) | (uint64_t)(k - mx_doff[u]));
                }
                std::sort(keys.begin(), keys.end());
                int64_t w = mx_doff[u];
                for (uint64_t key : keys) {
                    far[w] = (int)(key >> 32);
                    fent[w] = (int)(key & 0xffffffffu);
                    fnear[w] = mx_dflag[mx_doff[u] + fent[w]];
                    w++;
                }
                far_end[u] = w;
            }
        }
        pt.mark("plan: symmetric: sorted partners");
        // rev[j]: where the partner's sorted list holds this unit's leaf (-1:
        // nowhere, the entry stays one-directional)
        hvec<int64_t> rev(ne);
        std::vector<int64_t> poff0(NU + 1, 0), poff1(NU + 1, 0), ioff(NU + 1, 0);
#pragma omp parallel for schedule(static)
        for (int u = 0; u < NU; u++)
            for (int64_t j = mx_doff[u]; j < far_end[u]; j++) rev[j] = -1;
        // the head of each pair (A < B) looks itself up in B's list and links
        // both entries; every entry is written by one head at most
#pragma omp parallel for schedule(static)
        for (int u = 0; u < NU; u++) {
            const int A = T.leaves[u];
            for (int64_t j = mx_doff[u]; j < far_end[u]; j++) {
                const int B = far[j], ub = unit_of[B];
                if (B < A) continue;
                const int *b0 = far.data() + mx_doff[ub], *b1 = far.data() + far_end[ub];
                const int *it = std::lower_bound(b0, b1, A);
                if (it != b1 && *it == A) {
                    const int64_t q = it - far.data();
                    rev[j] = q;
                    rev[q] = j;
                }
            }
        }
        int64_t npaired = 0;       // entries in a pair, whichever shard evaluates it
#pragma omp parallel for schedule(static) reduction(+ : npaired)
        for (int u = 0; u < NU; u++) {
            const int A = T.leaves[u];
            int64_t heads[2] = {0, 0}, all = 0;
            for (int64_t j = mx_doff[u]; j < far_end[u]; j++)
                if (rev[j] >= 0) {
                    npaired++;
                    const bool head = A < far[j];
                    if (head ? owned[u] : owned[unit_of[far[j]]]) all++;
                    heads[fnear[j]] += head && owned[u] ? 1 : 0;
                }
            poff0[u + 1] = heads[0];
            poff1[u + 1] = heads[1];
            ioff[u + 1] = all;
        }
        for (int u = 0; u < NU; u++) {
            poff0[u + 1] += poff0[u];
            ioff[u + 1] += ioff[u];
        }
        sym_far_pairs = poff0[NU];
        poff1[0] = sym_far_pairs;
        for (int u = 0; u < NU; u++) poff1[u + 1] += poff1[u];
        pt.mark("plan: symmetric: reverse look-ups");
        const int64_t npairs = poff1[NU];
        if (npaired > 0) {
            // pairs headed by each unit, and the pair number of each head entry
            sym_pairs.resize((size_t)npairs);
            hvec<int64_t> pid(ne);
            std::vector<int64_t> usz0(NU + 1, 0), usz1(NU + 1, 0);
#pragma omp parallel for schedule(static)
            for (int u = 0; u < NU; u++) {
                const int A = T.leaves[u];
                int64_t p[2] = {poff0[u], poff1[u]}, sz[2] = {0, 0};
                for (int64_t j = mx_doff[u]; j < far_end[u]; j++)
                    if (rev[j] >= 0 && A < far[j] && owned[u]) {
                        const int g = fnear[j];
                        pid[j] = p[g];
                        sym_pairs[p[g]++] = make_int2(A, far[j]);
                        sz[g] += S.numpar[A] + S.numpar[far[j]];
                    }
                usz0[u + 1] = sz[0];
                usz1[u + 1] = sz[1];
            }
            for (int u = 0; u < NU; u++) usz0[u + 1] += usz0[u];
            usz1[0] = usz0[NU];
            for (int u = 0; u < NU; u++) usz1[u + 1] += usz1[u];
            sym_total = usz1[NU];
            // each pair's partial sums: A's particles, then B's
            sym_slot.resize((size_t)npairs);
#pragma omp parallel for schedule(static)
            for (int u = 0; u < NU; u++) {
                const int64_t pb[2] = {poff0[u], poff1[u]}, pe[2] = {poff0[u + 1], poff1[u + 1]};
                const int64_t sb[2] = {usz0[u], usz1[u]};
                for (int g = 0; g < 2; g++) {
                    int64_t s = sb[g];
                    for (int64_t p = pb[g]; p < pe[g]; p++) {
                        sym_slot[p] = s;
                        s += S.numpar[sym_pairs[p].x] + S.numpar[sym_pairs[p].y];
                    }
                }
            }
            // per leaf the slices addressed to it, in partner order: its own
            // side of the pairs it heads, the B side of the pairs headed by
            // a partner (found through the partner's entry for this leaf)
            sym_in_off = ioff;
            sym_in_slot.resize((size_t)ioff[NU]);
            hvec<unsigned char> drop(ne);
#pragma omp parallel for schedule(static)
            for (int u = 0; u < NU; u++) {
                const int A = T.leaves[u];
                int64_t w = ioff[u];
                std::fill(drop.begin() + mx_doff[u], drop.begin() + mx_doff[u + 1], (unsigned char)0);
                for (int64_t j = mx_doff[u]; j < far_end[u]; j++) {
                    if (rev[j] < 0) continue;
                    const int B = far[j];
                    // both directions leave the lists; only this shard's pairs are gathered
                    drop[mx_doff[u] + fent[j]] = 1;
                    if (!(A < B ? owned[u] : owned[unit_of[B]])) continue;
                    sym_in_slot[w++] = A < B ? sym_slot[pid[j]] : sym_slot[pid[rev[j]]] + S.numpar[B];
                }
            }
            pt.mark("plan: symmetric: pairs and slots");
            // both directions leave the per-target near-field lists
            std::vector<int64_t> noff(NU + 1, 0);
#pragma omp parallel for schedule(static)
            for (int u = 0; u < NU; u++) {
                int64_t kept = 0;
                for (int64_t k = mx_doff[u]; k < mx_doff[u + 1]; k++) kept += !drop[k];
                noff[u + 1] = kept;
            }
            for (int u = 0; u < NU; u++) noff[u + 1] += noff[u];
            hvec<int> nidx((size_t)noff[NU]);
            hvec<unsigned char> nflag((size_t)noff[NU]);
#pragma omp parallel for schedule(static)
            for (int u = 0; u < NU; u++) {
                int64_t w = noff[u];
                for (int64_t k = mx_doff[u]; k < mx_doff[u + 1]; k++)
                    if (!drop[k]) { nidx[w] = mx_didx[k]; nflag[w] = mx_dflag[k]; w++; }
            }
            mx_doff.swap(noff);
            mx_didx.swap(nidx);
            mx_dflag.swap(nflag);
        }
    }
    pt.mark("plan: symmetric near-field pairs");
    // Hermite upward pass: particle chunks of every source node
    std::vector<bt::HermChunk> hchunks;
    std::vector<int3> hred;
    int hslots = 0;
    if (herm && need_src_clusters) hslots = bt::hermite_chunks(S.n, S.ibeg, S.numpar, hchunks, hred);
    bt::HermChunk *d_hchunks = nullptr;
    int3 *d_hred = nullptr;
    double *d_hpartial = nullptr;

    // device layout
    double *d_sx, *d_sy, *d_sz, *d_sq, *d_tx, *d_ty, *d_tz, *d_pot, *d_sgrid, *d_tgrid, *d_slen, *d_tlen, *d_ww;
    double *d_Q = nullptr, *d_Phi = nullptr;
    int *d_sibeg, *d_snum, *d_snch, *d_sch, *d_sleaves, *d_slvl;
    int *d_tibeg, *d_tnum, *d_tnch, *d_tch, *d_tpar, *d_tleaves, *d_tlvl;
    int64_t *d_aoff, *d_doff, *d_ccoff, *d_cpoff;
    int *d_aidx, *d_didx, *d_ccidx, *d_cpidx;
    int2 *d_evitems, *d_griditems, *d_l2pitems;
    int *d_order;
    double *d_out;
    pt.mark("plan: Hermite chunks, device layout");
    Layout L;
    if (dp) {
        d_sx = (double *)dp->sx; d_sy = (double *)dp->sy; d_sz = (double *)dp->sz; d_sq = (double *)dp->sq;
        d_tx = (double *)dp->tx; d_ty = (double *)dp->ty; d_tz = (double *)dp->tz; d_order = (int *)dp->order;
    } else {
        L.add(&d_sx, ns); L.add(&d_sy, ns); L.add(&d_sz, ns); L.add(&d_sq, ns);
        L.add(&d_tx, nt); L.add(&d_ty, nt); L.add(&d_tz, nt); L.add(&d_order, nt);
    }
    L.add(&d_pot, nt);
    L.add(&d_sgrid, sgrid.size()); L.add(&d_tgrid, tgrid.size());
    L.add(&d_slen, slen.size()); L.add(&d_tlen, tlen.size()); L.add(&d_ww, BT_MAX_DEGREE + 1);
    if (need_src_clusters) L.add(&d_Q, (size_t)S.n * P * nq);
    if (need_tgt_grids) L.add(&d_Phi, (size_t)T.n * P * nq);
    L.add(&d_sibeg, S.n); L.add(&d_snum, S.n); L.add(&d_snch, S.n); L.add(&d_sch, 8 * (size_t)S.n);
    L.add(&d_sleaves, S.nleaves); L.add(&d_slvl, S.lvl_off ? S.lvl_off[S.max_depth] : 0);
    L.add(&d_tibeg, T.n); L.add(&d_tnum, T.n); L.add(&d_tnch, T.n); L.add(&d_tch, 8 * (size_t)T.n);
    L.add(&d_tpar, T.n); L.add(&d_tleaves, T.nleaves); L.add(&d_tlvl, T.lvl_off ? T.lvl_off[T.max_depth] : 0);
    L.add(&d_aoff, pl.t_approx.rows + 1); L.add(&d_aidx, pl.t_approx.off[pl.t_approx.rows]);
    L.add(&d_doff, pl.t_direct.rows + 1); L.add(&d_didx, pl.t_direct.off[pl.t_direct.rows]);
    L.add(&d_ccoff, pl.g_cc.rows + 1); L.add(&d_ccidx, pl.g_cc.off[pl.g_cc.rows]);
    L.add(&d_cpoff, pl.g_cp.rows + 1); L.add(&d_cpidx, pl.g_cp.off[pl.g_cp.rows]);
    L.add(&d_evitems, ev_items.size()); L.add(&d_griditems, grid_items.size()); L.add(&d_l2pitems, l2p_items.size());
    L.add(&d_out, nt);
    int *d_queue;           // work-queue counters of the two evaluation kernels, then the error flag
    L.add(&d_queue, 3);
    // subtraction: target charges and source weights in tree order, q*w,
    // the weight proxies and the weight field, a staging buffer for the
    // caller-order inputs, and the source order when the host built the tree
    double *d_tq = nullptr, *d_sw = nullptr, *d_qw = nullptr, *d_W = nullptr, *d_Phiw = nullptr, *d_ssin = nullptr;
    int *d_sordh = nullptr;
    if (ssm) {
        L.add(&d_tq, nt); L.add(&d_sw, ns); L.add(&d_qw, ns); L.add(&d_ssin, std::max(nt, ns));
        if (need_src_clusters) L.add(&d_W, (size_t)S.n * P * nq);
        if (need_tgt_grids) L.add(&d_Phiw, (size_t)T.n * P);
        if (!dp) L.add(&d_sordh, ns);
    }
    if (herm && need_src_clusters) {
        L.add(&d_hchunks, hchunks.size());
        L.add(&d_hred, hred.size());
        L.add(&d_hpartial, (size_t)hslots * 8 * P);
    }
    float4 *d_spos = nullptr, *d_tpos = nullptr;
    float *d_Q32 = nullptr;
    double *d_sctr = nullptr, *d_tctr = nullptr;
    int64_t *d_mxdoff = nullptr, *d_mxcpoff = nullptr;
    int *d_mxdidx = nullptr, *d_mxcpidx = nullptr;
    unsigned char *d_mxdflag = nullptr, *d_adeg = nullptr;
    double *d_xgrid[BT_MAX_DEGREE + 1] = {}, *d_xQ[BT_MAX_DEGREE + 1] = {};
    double *d_srad = nullptr, *d_trad = nullptr;
    float *d_xQ32[BT_MAX_DEGREE + 1] = {};
    int *d_xleaves[BT_MAX_DEGREE + 1] = {}, *d_xlvl[BT_MAX_DEGREE + 1] = {};
    int2 *d_sym_pairs = nullptr;
    int64_t *d_sym_slot = nullptr, *d_sym_in_off = nullptr, *d_sym_in_slot = nullptr;
    float *d_sym_partial = nullptr;
    double *d_sbox = nullptr;
    if (mixed) {
        L.add(&d_spos, ns); L.add(&d_tpos, nt);
        if (need_src_clusters) L.add(&d_Q32, (size_t)S.n * P * nq);
        L.add(&d_sctr, sctr.size()); L.add(&d_tctr, tctr.size());
        L.add(&d_mxdoff, mx_doff.size()); L.add(&d_mxdidx, mx_didx.size()); L.add(&d_mxdflag, mx_dflag.size());
        L.add(&d_mxcpoff, mx_cpoff.size()); L.add(&d_mxcpidx, mx_cpidx.size());
        if (pl.a_deg) L.add(&d_adeg, n_approx);
        L.add(&d_srad, S.n); L.add(&d_trad, T.n);
        if ((int64_t)sym_pairs.size() > sym_far_pairs) L.add(&d_sbox, 6 * (size_t)S.n);
        if (!sym_pairs.empty()) {
            L.add(&d_sym_pairs, sym_pairs.size()); L.add(&d_sym_slot, sym_slot.size());
            L.add(&d_sym_in_off, sym_in_off.size()); L.add(&d_sym_in_slot, sym_in_slot.size());
            L.add(&d_sym_partial, (size_t)sym_total);
        }
        for (size_t i = 0; i < xdeg.size(); i++) {
            size_t Pd = (size_t)(xdeg[i] + 1) * (xdeg[i] + 1) * (xdeg[i] + 1);
            L.add(&d_xgrid[i], xgrid[i].size());
            L.add(&d_xQ[i], (size_t)S.n * Pd);
            L.add(&d_xQ32[i], (size_t)S.n * Pd);
            L.add(&d_xleaves[i], xleaves[i].size());
            L.add(&d_xlvl[i], xlvl[i].size());
        }
    }

    if (!arena.reserve(L.total())) {
        if (arena.fixed) {
            set_err("this call needs %zu bytes of device scratch; the static scratch holds %zu", L.total(), arena.cap);
            return BT_ERR_PARAM;
        }
        set_err("device allocation of %zu bytes failed", L.total());
        return BT_ERR_CUDA;
    }
    L.bind(arena);

    double t_setup = now_ms();
    {
#define UP(dst, src, cnt)                                                                              \
    if ((cnt) > 0) CK(cudaMemcpyAsync(dst, src, sizeof(*(src)) * (size_t)(cnt), cudaMemcpyHostToDevice, st))
        if (!dp) {
            UP(d_sx, pl.src.x, ns); UP(d_sy, pl.src.y, ns); UP(d_sz, pl.src.z, ns); UP(d_sq, pl.src.q, ns);
            UP(d_tx, pl.tgt.x, nt); UP(d_ty, pl.tgt.y, nt); UP(d_tz, pl.tgt.z, nt);
            UP(d_order, pl.tgt.order, nt);
        }
        UP(d_sgrid, sgrid.data(), sgrid.size()); UP(d_tgrid, tgrid.data(), tgrid.size());
        UP(d_slen, slen.data(), slen.size()); UP(d_tlen, tlen.data(), tlen.size());
        UP(d_ww, ww, n + 1);
        UP(d_sibeg, S.ibeg, S.n); UP(d_snum, S.numpar, S.n); UP(d_snch, S.nchild, S.n); UP(d_sch, S.child, 8 * (size_t)S.n);
        UP(d_sleaves, S.leaves, S.nleaves);
        if (S.lvl_off) UP(d_slvl, S.lvl_nodes, S.lvl_off[S.max_depth]);
        UP(d_tibeg, T.ibeg, T.n); UP(d_tnum, T.numpar, T.n); UP(d_tnch, T.nchild, T.n); UP(d_tch, T.child, 8 * (size_t)T.n);
        UP(d_tpar, T.parent, T.n); UP(d_tleaves, T.leaves, T.nleaves);
        if (T.lvl_off) UP(d_tlvl, T.lvl_nodes, T.lvl_off[T.max_depth]);
        UP(d_aoff, pl.t_approx.off, pl.t_approx.rows + 1); UP(d_aidx, pl.t_approx.idx, pl.t_approx.off[pl.t_approx.rows]);
        UP(d_doff, pl.t_direct.off, pl.t_direct.rows + 1); UP(d_didx, pl.t_direct.idx, pl.t_direct.off[pl.t_direct.rows]);
        UP(d_ccoff, pl.g_cc.off, pl.g_cc.rows + 1); UP(d_ccidx, pl.g_cc.idx, pl.g_cc.off[pl.g_cc.rows]);
        UP(d_cpoff, pl.g_cp.off, pl.g_cp.rows + 1); UP(d_cpidx, pl.g_cp.idx, pl.g_cp.off[pl.g_cp.rows]);
        UP(d_evitems, ev_items.data(), ev_items.size());
        if (herm && need_src_clusters) {
            UP(d_hchunks, hchunks.data(), hchunks.size());
            UP(d_hred, hred.data(), hred.size());
        }
        UP(d_griditems, grid_items.data(), grid_items.size());
        UP(d_l2pitems, l2p_items.data(), l2p_items.size());
        if (ssm) {
            const cudaMemcpyKind kin = ss->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
            const int *sorder = dp ? dp->sorder : d_sordh;
            if (!dp) UP(d_sordh, pl.src.order, ns);
            if (nt > 0) CK(cudaMemcpyAsync(d_ssin, ss->tq, sizeof(double) * (size_t)nt, kin, st));
            bt::launch_gather(nt, d_order, d_ssin, d_tq, st);
            if (ns > 0) CK(cudaMemcpyAsync(d_ssin, ss->sw, sizeof(double) * (size_t)ns, kin, st));
            bt::launch_gather(ns, sorder, d_ssin, d_sw, st);
            bt::launch_mul(ns, d_sq, d_sw, d_qw, st);
            launches += 3;
        }
        if (mixed) {
            UP(d_sctr, sctr.data(), sctr.size()); UP(d_tctr, tctr.data(), tctr.size());
            UP(d_mxdoff, mx_doff.data(), mx_doff.size()); UP(d_mxdidx, mx_didx.data(), mx_didx.size());
            UP(d_mxdflag, mx_dflag.data(), mx_dflag.size());
            std::vector<double> sbox;
            if (d_sbox) {
                sbox.resize(6 * (size_t)S.n);
                for (int i = 0; i < S.n; i++) {
                    double *b = sbox.data() + 6 * (size_t)i;
                    b[0] = S.x0[i]; b[1] = S.x1[i]; b[2] = S.y0[i]; b[3] = S.y1[i]; b[4] = S.z0[i]; b[5] = S.z1[i];
                }
                UP(d_sbox, sbox.data(), sbox.size());
            }
            if (!sym_pairs.empty()) {
                UP(d_sym_pairs, sym_pairs.data(), sym_pairs.size()); UP(d_sym_slot, sym_slot.data(), sym_slot.size());
                UP(d_sym_in_off, sym_in_off.data(), sym_in_off.size()); UP(d_sym_in_slot, sym_in_slot.data(), sym_in_slot.size());
            }
            if (pl.a_deg) UP(d_adeg, pl.a_deg, n_approx);
            UP(d_srad, S.rad, S.n); UP(d_trad, T.rad, T.n);
            for (size_t i = 0; i < xdeg.size(); i++) {
                UP(d_xgrid[i], xgrid[i].data(), xgrid[i].size());
                UP(d_xleaves[i], xleaves[i].data(), xleaves[i].size());
                UP(d_xlvl[i], xlvl[i].data(), xlvl[i].size());
            }
            UP(d_mxcpoff, mx_cpoff.data(), mx_cpoff.size()); UP(d_mxcpidx, mx_cpidx.data(), mx_cpidx.size());
        }
#undef UP
        cudaEvent_t *ev = ctx->ev;
        DevPlan v;
        v.mixed = mixed; v.herm = herm; v.need_src_clusters = need_src_clusters; v.need_tgt_grids = need_tgt_grids;
        v.queue = shape.queue;
        v.tpt = shape.tpt;
        v.tile = shape.tile;
        v.tc_up = shape.tc_up && mixed;
        v.sharded = shape.nshards > 1;
        v.fp64_tb = fp64_tb;
        v.base_full = pl.a_deg == nullptr;
        v.sym_npairs = (int)sym_pairs.size();
        v.sym_far_pairs = (int)sym_far_pairs;
        v.d_sbox = d_sbox;
        v.d_sym_pairs = d_sym_pairs; v.d_sym_slot = d_sym_slot; v.d_sym_in_off = d_sym_in_off;
        v.d_sym_in_slot = d_sym_in_slot; v.d_sym_partial = d_sym_partial;
        v.n = n; v.P = P; v.ns = ns; v.nt = nt; v.max_np1 = max_np1; v.kernel = o.kernel; v.kp = o.kp;
        v.S_n = S.n; v.S_nleaves = S.nleaves; v.S_max_depth = S.max_depth;
        v.T_n = T.n; v.T_nleaves = T.nleaves; v.T_max_depth = T.max_depth;
        if (S.lvl_off) v.S_lvl_off.assign(S.lvl_off, S.lvl_off + S.max_depth + 1);
        else v.S_lvl_off.assign(S.max_depth + 1, 0);
        if (T.lvl_off) v.T_lvl_off.assign(T.lvl_off, T.lvl_off + T.max_depth + 1);
        else v.T_lvl_off.assign(T.max_depth + 1, 0);
        v.xdeg = xdeg;
        v.n_grid_items = (int)grid_items.size(); v.n_ev_items = (int)ev_items.size(); v.n_l2p_items = (int)l2p_items.size();
        v.d_hchunks = d_hchunks; v.d_hred = d_hred; v.d_hpartial = d_hpartial;
        v.ss = ssm; v.kp2 = o.kp2; v.ss_c = ssm ? bt::ss_correction_constant(o.kernel, o.kp) : 0.0;
        v.d_tq = d_tq; v.d_sw = d_sw; v.d_qw = d_qw; v.d_W = d_W; v.d_Phiw = d_Phiw;
        v.n_hchunks = (int)hchunks.size(); v.n_hred = (int)hred.size();
        v.d_sx = d_sx;
        v.d_sy = d_sy;
        v.d_sz = d_sz;
        v.d_sq = d_sq;
        v.d_tx = d_tx;
        v.d_ty = d_ty;
        v.d_tz = d_tz;
        v.d_pot = d_pot;
        v.d_sgrid = d_sgrid;
        v.d_tgrid = d_tgrid;
        v.d_slen = d_slen;
        v.d_tlen = d_tlen;
        v.d_ww = d_ww;
        v.d_Q = d_Q;
        v.d_Phi = d_Phi;
        v.d_srad = d_srad;
        v.d_trad = d_trad;
        v.d_sctr = d_sctr;
        v.d_tctr = d_tctr;
        v.d_sibeg = d_sibeg;
        v.d_snum = d_snum;
        v.d_snch = d_snch;
        v.d_sch = d_sch;
        v.d_sleaves = d_sleaves;
        v.d_slvl = d_slvl;
        v.d_tibeg = d_tibeg;
        v.d_tnum = d_tnum;
        v.d_tnch = d_tnch;
        v.d_tch = d_tch;
        v.d_tpar = d_tpar;
        v.d_tleaves = d_tleaves;
        v.d_tlvl = d_tlvl;
        v.d_aidx = d_aidx;
        v.d_didx = d_didx;
        v.d_ccidx = d_ccidx;
        v.d_cpidx = d_cpidx;
        v.d_order = d_order;
        v.d_queue = d_queue;
        v.d_err = d_queue + 2;
        v.d_mxdidx = d_mxdidx;
        v.d_mxcpidx = d_mxcpidx;
        v.d_aoff = d_aoff;
        v.d_doff = d_doff;
        v.d_ccoff = d_ccoff;
        v.d_cpoff = d_cpoff;
        v.d_mxdoff = d_mxdoff;
        v.d_mxcpoff = d_mxcpoff;
        v.d_evitems = d_evitems;
        v.d_griditems = d_griditems;
        v.d_l2pitems = d_l2pitems;
        v.d_spos = d_spos;
        v.d_tpos = d_tpos;
        v.d_Q32 = d_Q32;
        v.d_mxdflag = d_mxdflag;
        v.d_adeg = d_adeg;
        for (int k = 0; k <= BT_MAX_DEGREE; k++) {
            v.d_xgrid[k] = d_xgrid[k]; v.d_xQ[k] = d_xQ[k]; v.d_xQ32[k] = d_xQ32[k];
            v.d_xleaves[k] = d_xleaves[k]; v.d_xlvl[k] = d_xlvl[k];
        }
        for (size_t i = 0; i < xdeg.size(); i++) v.xleaf_n.push_back((int)xleaves[i].size());
        v.xlvl_off = xlvl_off;
        if (dv_out) {
            *dv_out = v;
            dv_out->d_out = d_out;
        }
        if (!execute) {
            CK(cudaStreamSynchronize(st));
            goto done;
        }
        pt.mark("plan: device arrays and uploads");
        rc = issue_plan(v, st, ev, out_on_device ? out : d_out, launches, false, &ctx->fk);
        if (rc != BT_OK) goto done;
        if (!out_on_device && nt > 0)
            CK(cudaMemcpyAsync(out, d_out, sizeof(double) * nt, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        rc = check_device_error(v, st);
        if (rc != BT_OK) goto done;
        pt.mark("evaluation (device, synchronised)");
        g_launches += launches;
        if (rep) {
            float a = 0, b = 0, c = 0, d = 0;
            cudaEventElapsedTime(&a, ev[0], ev[1]);
            cudaEventElapsedTime(&b, ev[1], ev[2]);
            cudaEventElapsedTime(&c, ev[2], ev[3]);
            cudaEventElapsedTime(&d, ev[3], ev[4]);
            cudaGetLastError();
            rep->ms_upward = a;
            rep->ms_compute = b + c;
            rep->ms_downward = d;
            rep->ms_eval_kernel = c;
            rep->kernel_launches = (int)launches;
            long long symw = 0;
            for (const int2 &pr : sym_pairs) symw += 2LL * S.numpar[pr.x] * S.numpar[pr.y];
            rep->sym_ptwise = symw;
            rep->source_nodes = S.n;
            rep->target_nodes = T.n;
            double tend = now_ms();
            rep->ms_transfer = (tend - t_setup) - (a + b + c + d);
            rep->ms_setup += t_setup - t0;      // host preparation of the device arrays
            rep->ms_total += tend - t0;
        }
    }
done:
    return rc;
}

// ---------------------------------------------------------------------------
// Learned degree selection (particle-cluster interactions, mixed path)
// ---------------------------------------------------------------------------
std::vector<float> g_selector;      // installed MLP weights (bt_selector_set), process-wide
std::mutex g_selector_mu;
// The selection's error share: every interaction (target, cluster entry) of
// a system may contribute SELECT_SHARE * tol * sqrt(sum_t phi_t^2 / sum_t N_t)
// in absolute terms, phi_t^2 estimated per target leaf at one sampled
// target, N_t its cluster entries (bt::launch_select_share), so that the
// system's relative L2 error stays below the tolerance; calibrated across
// eight workloads.  BARYTREE_B200_SELECT_SHARE overrides it (calibration).
constexpr double SELECT_SHARE = 0.35;

double select_share()
{
    const char *e = getenv("BARYTREE_B200_SELECT_SHARE");
    return e ? atof(e) : SELECT_SHARE;
}

void node_geometry(const bt_tree &t, std::vector<double> &ctr, std::vector<double> &rad)
{
    ctr.resize(3 * (size_t)t.n);
    rad.resize(t.n);
    for (int i = 0; i < t.n; i++) {
        ctr[3 * i] = t.xm[i]; ctr[3 * i + 1] = t.ym[i]; ctr[3 * i + 2] = t.zm[i];
        rad[i] = t.rad[i];
    }
}

// Predict the error of every particle-cluster entry at every degree, choose
// the lowest degree under the system's error share (or direct evaluation),
// and rewrite the plan's target-leaf lists accordingly.
int select_degrees(DeviceCtx *ctx, Arena &arena, bt_plan &pl, double tol, const DevParts *dp = nullptr)
{
    std::vector<float> w;
    {
        std::lock_guard<std::mutex> lk(g_selector_mu);
        w = g_selector;
    }
    if ((int)w.size() != bt::MLP_NWEIGHTS) {
        set_err("no degree selector installed (bt_selector_set)");
        return BT_ERR_PARAM;
    }
    const bt_tree &S = pl.st, &T = pl.tt;
    PhaseTimer pt;
    const int64_t ne = pl.t_approx.off[pl.t_approx.rows];
    std::vector<unsigned char> choice(ne > 0 ? ne : 1);
    cudaStream_t st = ctx->stream;
    int rc = BT_OK;
    if (ne > 0) {
        std::vector<double> sctr, srad, tctr, trad;
        node_geometry(S, sctr, srad);
        node_geometry(T, tctr, trad);
        double *d_sq, *d_mom, *d_sctr, *d_tctr, *d_srad, *d_trad;
        int *d_sibeg, *d_snum, *d_tnum, *d_idx, *d_unit, *d_snch, *d_sch, *d_sleaves, *d_slvl;
        int64_t *d_off;
        float *d_feat, *d_w, *d_pred;
        unsigned char *d_choice;
        pt.mark("selection: node geometry (host)");
        Layout L;
        if (dp) d_sq = (double *)dp->sq;
        else L.add(&d_sq, pl.src.n);
        L.add(&d_mom, 2 * (size_t)S.n); L.add(&d_sctr, sctr.size()); L.add(&d_tctr, tctr.size());
        L.add(&d_srad, srad.size()); L.add(&d_trad, trad.size()); L.add(&d_sibeg, S.n); L.add(&d_snum, S.n);
        L.add(&d_snch, S.n); L.add(&d_sch, 8 * (size_t)S.n); L.add(&d_sleaves, S.nleaves);
        L.add(&d_slvl, S.lvl_off ? S.lvl_off[S.max_depth] : 0);
        L.add(&d_tnum, T.n); L.add(&d_idx, ne); L.add(&d_unit, T.nleaves); L.add(&d_off, pl.t_approx.rows + 1);
        L.add(&d_feat, (size_t)ne * bt::MLP_IN); L.add(&d_w, w.size());
        L.add(&d_pred, (size_t)ne * bt::MLP_OUT); L.add(&d_choice, ne);
        int *d_mlperr;          // set by the MLP kernel if a bounded wait expired
        L.add(&d_mlperr, 1);
        // the error share: near-field lists, the target leaves' first
        // particles, per-unit sums, one share per system; the particles in
        // tree order (on the device already after a GPU tree build)
        const double share_c = select_share();
        const int64_t nd = pl.t_direct.off[pl.t_direct.rows];
        const int nsys = T.nroots;
        int64_t *d_doff;
        int *d_didx, *d_tibeg, *d_sysoff;
        double *d_usum;
        float *d_share;
        L.add(&d_doff, pl.t_direct.rows + 1); L.add(&d_didx, nd > 0 ? nd : 1); L.add(&d_tibeg, T.n);
        L.add(&d_usum, 2 * (size_t)pl.t_approx.rows); L.add(&d_share, nsys); L.add(&d_sysoff, nsys + 1);
        const double *px = dp ? dp->sx : nullptr, *py = dp ? dp->sy : nullptr, *pz = dp ? dp->sz : nullptr;
        const double *ptx = dp ? dp->tx : nullptr, *pty = dp ? dp->ty : nullptr, *ptz = dp ? dp->tz : nullptr;
        double *hx = nullptr, *hy = nullptr, *hz = nullptr, *htx = nullptr, *hty = nullptr, *htz = nullptr;
        if (!dp) {
            L.add(&hx, pl.src.n); L.add(&hy, pl.src.n); L.add(&hz, pl.src.n);
            L.add(&htx, pl.tgt.n); L.add(&hty, pl.tgt.n); L.add(&htz, pl.tgt.n);
        }
        if (!arena.reserve(L.total())) {
            set_err(arena.fixed ? "degree selection needs more scratch than the static array holds"
                                : "device allocation failed");
            return arena.fixed ? BT_ERR_PARAM : BT_ERR_CUDA;
        }
        L.bind(arena);
        {
#define UP(dst, src, cnt) CK(cudaMemcpyAsync(dst, src, sizeof(*(src)) * (size_t)(cnt), cudaMemcpyHostToDevice, st))
            if (!dp) UP(d_sq, pl.src.q, pl.src.n);
            UP(d_sctr, sctr.data(), sctr.size()); UP(d_tctr, tctr.data(), tctr.size());
            UP(d_srad, srad.data(), srad.size()); UP(d_trad, trad.data(), trad.size());
            UP(d_sibeg, S.ibeg, S.n); UP(d_snum, S.numpar, S.n); UP(d_tnum, T.numpar, T.n);
            UP(d_snch, S.nchild, S.n); UP(d_sch, S.child, 8 * (size_t)S.n); UP(d_sleaves, S.leaves, S.nleaves);
            if (S.lvl_off && S.lvl_off[S.max_depth] > 0) UP(d_slvl, S.lvl_nodes, S.lvl_off[S.max_depth]);
            UP(d_idx, pl.t_approx.idx, ne); UP(d_unit, T.leaves, T.nleaves);
            UP(d_off, pl.t_approx.off, pl.t_approx.rows + 1); UP(d_w, w.data(), w.size());
#undef UP
            bt::MomentTree mt{S.n, S.nleaves, S.max_depth, d_sleaves, d_sibeg, d_snum, d_snch, d_sch, d_slvl, S.lvl_off};
            long long launches = bt::launch_node_moments(mt, d_sq, d_mom, st);
            bt::FeatureArgs fa;
            fa.units = pl.t_approx.rows; fa.off = d_off; fa.idx = d_idx; fa.unit_node = d_unit;
            fa.t_ctr = d_tctr; fa.s_ctr = d_sctr; fa.t_rad = d_trad; fa.s_rad = d_srad; fa.s_mom = d_mom;
            fa.t_numpar = d_tnum; fa.s_numpar = d_snum;
            bt::launch_features(fa, ne, d_feat, st);
            launches++;
            CK(cudaMemsetAsync(d_mlperr, 0, sizeof(int), st));
            bt::mlp_infer_tc(d_w, ne, d_feat, d_pred, d_mlperr, st);
            launches++;
            CK(cudaMemcpyAsync(d_doff, pl.t_direct.off, sizeof(int64_t) * (pl.t_direct.rows + 1),
                               cudaMemcpyHostToDevice, st));
            if (nd > 0) CK(cudaMemcpyAsync(d_didx, pl.t_direct.idx, sizeof(int) * nd, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_tibeg, T.ibeg, sizeof(int) * T.n, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_sysoff, T.leaf_off, sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice, st));
            if (!dp) {
                const double *src[6] = {pl.src.x, pl.src.y, pl.src.z, pl.tgt.x, pl.tgt.y, pl.tgt.z};
                double *dst[6] = {hx, hy, hz, htx, hty, htz};
                for (int k = 0; k < 6; k++)
                    CK(cudaMemcpyAsync(dst[k], src[k], sizeof(double) * (k < 3 ? pl.src.n : pl.tgt.n),
                                       cudaMemcpyHostToDevice, st));
                px = hx; py = hy; pz = hz; ptx = htx; pty = hty; ptz = htz;
            }
            bt::launch_select_share(fa, nsys, d_sysoff, d_tibeg, d_doff, d_didx, d_sibeg, px, py, pz, d_sq, ptx, pty,
                                    ptz, share_c * tol, ne, d_pred, d_feat, d_usum, d_share, d_choice, st);
            launches += 3;
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(choice.data(), d_choice, ne, cudaMemcpyDeviceToHost, st));
            int mlperr = 0;
            CK(cudaMemcpyAsync(&mlperr, d_mlperr, sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            g_launches += launches;
            if (mlperr) {
                set_err("the degree selector's tensor-core kernel timed out waiting for its MMAs");
                return BT_ERR_TIMEOUT;
            }
        }
    }
    pt.mark("selection: features + MLP (GPU)");
    {
        // rewrite the target-leaf lists: chosen degree per kept entry, direct
        // evaluation for the rest (appended to the direct list)
        const int rows = pl.t_approx.rows;
        int64_t *aoff = (int64_t *)malloc(sizeof(int64_t) * (rows + 1));
        int64_t *doff = (int64_t *)malloc(sizeof(int64_t) * (rows + 1));
        aoff[0] = doff[0] = 0;
        // per row: entries kept as clusters and entries moved to the direct list
#pragma omp parallel for schedule(static)
        for (int u = 0; u < rows; u++) {
            int64_t na = 0, nd = pl.t_direct.off[u + 1] - pl.t_direct.off[u];
            for (int64_t k = pl.t_approx.off[u]; k < pl.t_approx.off[u + 1]; k++) {
                if (choice[k] == bt::MLP_PP) nd++;
                else na++;
            }
            aoff[u + 1] = na;
            doff[u + 1] = nd;
        }
        for (int u = 0; u < rows; u++) {
            aoff[u + 1] += aoff[u];
            doff[u + 1] += doff[u];
        }
        // the new lists, filled in parallel straight into their final arrays
        int *aidx = (int *)malloc(sizeof(int) * ((size_t)aoff[rows] + 1));
        int *didx = (int *)malloc(sizeof(int) * ((size_t)doff[rows] + 1));
        unsigned char *adeg = (unsigned char *)malloc((size_t)aoff[rows] + 1);
        long long hist[14] = {};
#pragma omp parallel
        {
            long long h[14] = {};
#pragma omp for schedule(static)
            for (int u = 0; u < rows; u++) {
                int64_t a = aoff[u], d = doff[u];
                for (int64_t k = pl.t_approx.off[u]; k < pl.t_approx.off[u + 1]; k++) {
                    h[choice[k] == bt::MLP_PP ? 13 : choice[k]]++;
                    if (choice[k] == bt::MLP_PP) didx[d++] = pl.t_approx.idx[k];
                    else { aidx[a] = pl.t_approx.idx[k]; adeg[a++] = choice[k]; }
                }
                for (int64_t k = pl.t_direct.off[u]; k < pl.t_direct.off[u + 1]; k++) didx[d++] = pl.t_direct.idx[k];
            }
#pragma omp critical
            for (int i = 0; i < 14; i++) hist[i] += h[i];
        }
        for (int i = 0; i < 14; i++) pl.sel_hist[i] += hist[i];
        bt_csr_free(&pl.t_approx);
        bt_csr_free(&pl.t_direct);
        pl.t_approx.rows = pl.t_direct.rows = rows;
        pl.t_approx.off = aoff;
        pl.t_direct.off = doff;
        pl.t_approx.idx = aidx;
        pl.t_direct.idx = didx;
        free(pl.a_deg);
        pl.a_deg = adeg;
    }
    pt.mark("selection: list rewrite (host)");
done:
    return rc;
}

// Interaction counts after a learned selection (what the kernels evaluate).
void count_learned(const bt_plan &pl, bt_report *r)
{
    const bt_tree &S = pl.st, &T = pl.tt;
    long long pp = 0, pc = 0;
#pragma omp parallel for schedule(static) reduction(+ : pp, pc)
    for (int u = 0; u < T.nleaves; u++) {
        long long m = T.numpar[T.leaves[u]];
        for (int64_t k = pl.t_direct.off[u]; k < pl.t_direct.off[u + 1]; k++) pp += m * S.numpar[pl.t_direct.idx[k]];
        for (int64_t k = pl.t_approx.off[u]; k < pl.t_approx.off[u + 1]; k++) {
            long long d1 = pl.a_deg[k] + 1;
            pc += m * d1 * d1 * d1;
        }
    }
    r->pp_ptwise = pp;
    for (int i = 0; i < 14; i++) r->selected[i] = pl.sel_hist[i];
    r->pc_ptwise = pc;
    r->eval_flops = (long long)(pp * flops_per_eval(pl.prm, false) + pc * flops_per_eval(pl.prm, true));
}

// ---------------------------------------------------------------------------
// Static device scratch of the allocation-free entry point bt_eval_noalloc.
// In host code the symbol is only a host-side stand-in: its device address is
// looked up once per device (cudaGetSymbolAddress with that device current)
// and only that address is handed to kernels.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[BT_NOALLOC_SCRATCH_BYTES];

struct StaticScratch {
    bool ready = false;
    Arena arena;
};
StaticScratch g_static_scratch[16];

// Called with `device` current and its context lock held.
int static_scratch_arena(int device, Arena **out)
{
    StaticScratch &s = g_static_scratch[device];
    if (!s.ready) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr) {
            set_err("cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
            return BT_ERR_CUDA;
        }
        s.arena.base = (char *)ptr;
        s.arena.cap = BT_NOALLOC_SCRATCH_BYTES;
        s.arena.fixed = true;
        s.ready = true;
    }
    *out = &s.arena;
    return BT_OK;
}

// Checks the options and applies them to prm: precision, learned degree
// policy and its tolerance, dispatch of the mixed evaluation kernels.
int parse_options(const bt_options *opts, bt_params &prm, bool &learned, double &tol, EvalConfig &shape)
{
    if (opts && opts->precision != BT_PRECISION_FP64 && opts->precision != BT_PRECISION_MIXED) {
        set_err("invalid precision %d", opts->precision);
        return BT_ERR_PARAM;
    }
    prm.precision = opts ? opts->precision : BT_PRECISION_FP64;
    learned = opts && opts->degree_policy == BT_DEGREE_LEARNED;
    if (opts && opts->degree_policy != BT_DEGREE_FIXED && !learned) {
        set_err("invalid degree policy %d", opts->degree_policy);
        return BT_ERR_PARAM;
    }
    if (opts && opts->tree_build != BT_TREE_GPU && opts->tree_build != BT_TREE_HOST) {
        set_err("invalid tree build %d", opts->tree_build);
        return BT_ERR_PARAM;
    }
    if (opts && (opts->dispatch < BT_DISPATCH_AUTO || opts->dispatch > BT_DISPATCH_GRID)) {
        set_err("invalid dispatch %d", opts->dispatch);
        return BT_ERR_PARAM;
    }
    // Tile shape and dispatch: the device's autotuned shape for this kernel
    // and approximation (bt_autotune / bt_tuning_set), else the defaults.
    // Default dispatch: one block per work item.  Persistent blocks on a
    // device counter measured 2.5 % slower for the 16M clustered system
    // (cost-sorted items are already dispatched longest first by the block
    // scheduler).  An explicit dispatch option overrides the tuned one.
    if (opts && opts->upward != BT_UPWARD_AUTO && opts->upward != BT_UPWARD_FP64) {
        set_err("invalid upward %d", opts->upward);
        return BT_ERR_PARAM;
    }
    shape = tuned_shape(opts ? opts->device : 0, prm.kernel, prm.approx);
    shape.tc_up = !(opts && opts->upward == BT_UPWARD_FP64);
    if (opts && opts->symmetry != BT_SYMMETRY_AUTO && opts->symmetry != BT_SYMMETRY_OFF) {
        set_err("invalid symmetry %d", opts->symmetry);
        return BT_ERR_PARAM;
    }
    shape.sym = !(opts && opts->symmetry == BT_SYMMETRY_OFF);
    if (opts && opts->shard_count > 1) {
        if (opts->shard_index < 0 || opts->shard_index >= opts->shard_count) {
            set_err("shard index %d outside [0, %d)", opts->shard_index, opts->shard_count);
            return BT_ERR_PARAM;
        }
        shape.shard = opts->shard_index;
        shape.nshards = opts->shard_count;
    } else if (opts && opts->shard_count < 0) {
        set_err("invalid shard count %d", opts->shard_count);
        return BT_ERR_PARAM;
    }
    if (opts && opts->dispatch == BT_DISPATCH_QUEUE) shape.queue = true;
    if (opts && opts->dispatch == BT_DISPATCH_GRID) shape.queue = false;
    if (learned && (prm.precision != BT_PRECISION_MIXED || prm.ctype != PARTICLE_CLUSTER || prm.approx != LAGRANGE ||
                    prm.kernel != COULOMB)) {
        set_err("learned degree selection is provided for mixed precision, particle-cluster, Lagrange, Coulomb");
        return BT_ERR_UNSUPPORTED;
    }
    tol = (opts && opts->tolerance > 0) ? opts->tolerance : 1e-6;
    return BT_OK;
}

int eval_common(const Systems &sys, const double *tx, const double *ty, const double *tz, const double *sx,
                const double *sy, const double *sz, const double *sq, double *out, bt_params &prm,
                const bt_options *opts, bt_report *rep, bool use_static_scratch = false,
                const double *tq = nullptr, const double *sw = nullptr)
{
    g_err[0] = 0;
    const int64_t nt64 = sys.toff[sys.n], ns64 = sys.soff[sys.n];
    if (nt64 > INT_MAX || ns64 > INT_MAX) { set_err("more than 2^31-1 particles"); return BT_ERR_PARAM; }
    const int nt = (int)nt64, ns = (int)ns64;
    int rc = validate(nt, ns, tx, ty, tz, sx, sy, sz, sq, out, prm);
    if (rc != BT_OK) return rc;
    const bool out_dev = opts && opts->inputs_on_device;
    if (nt > 0 && !out_dev) memset(out, 0, sizeof(double) * (size_t)nt);
    if (rep) memset(rep, 0, sizeof(*rep));
    if (nt == 0) return BT_OK;
    if (ns == 0) {
        if (out_dev && cudaMemset(out, 0, sizeof(double) * (size_t)nt) != cudaSuccess) { set_err("cudaMemset failed"); return BT_ERR_CUDA; }
        return BT_OK;
    }
    int device = opts ? opts->device : 0;
    bool learned = false;
    EvalConfig shape;
    double tol = 1e-6;
    rc = parse_options(opts, prm, learned, tol, shape);
    if (rc != BT_OK) return rc;
    if (prm.sing == SUBTRACTION) {
        // Particles_Validate (src/particles/particles.c:170-193): subtraction
        // needs the target charges and source weights
        if (!tq || !sw) {
            set_err("singularity subtraction needs target charges and source weights");
            return BT_ERR_PARAM;
        }
        if (learned) {
            set_err("learned degree selection is not provided with singularity subtraction");
            return BT_ERR_UNSUPPORTED;
        }
    }
    DeviceCtx *ctx = nullptr;
    rc = get_ctx(device, &ctx);
    if (rc != BT_OK) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Arena *arena = &ctx->arena;
    if (use_static_scratch) {
        rc = static_scratch_arena(device, &arena);
        if (rc != BT_OK) return rc;
    }
    double t0 = now_ms();
    const bool on_dev = opts && opts->inputs_on_device;
    const bool gpu_tree = !use_static_scratch && !(opts && opts->tree_build == BT_TREE_HOST);
    bt_plan pl;
    memset(&pl, 0, sizeof pl);
    pl.prm = prm;
    DevParts dp;
    if (gpu_tree) {
        rc = build_plan_gpu(ctx, ctx->tree_arena, pl, sys, tx, ty, tz, sx, sy, sz, sq, on_dev, dp);
        if (rc != BT_OK) {
            bt_plan_free(&pl);
            return rc;
        }
    } else {
        std::vector<double> hbuf;
        if (on_dev) {
            // Device-resident inputs with the host tree build: bring the
            // coordinates over once.
            hbuf.resize((size_t)3 * nt + 4 * (size_t)ns);
            const double *src[7] = {tx, ty, tz, sx, sy, sz, sq};
            size_t cnt[7] = {(size_t)nt, (size_t)nt, (size_t)nt, (size_t)ns, (size_t)ns, (size_t)ns, (size_t)ns};
            double *dst = hbuf.data();
            const double *hp[7];
            for (int k = 0; k < 7; k++) {
                if (cudaMemcpyAsync(dst, src[k], sizeof(double) * cnt[k], cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) {
                    set_err("copy of device inputs failed");
                    return BT_ERR_CUDA;
                }
                hp[k] = dst;
                dst += cnt[k];
            }
            if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { set_err("copy of device inputs failed"); return BT_ERR_CUDA; }
            tx = hp[0]; ty = hp[1]; tz = hp[2]; sx = hp[3]; sy = hp[4]; sz = hp[5]; sq = hp[6];
        }
        build_plan(pl, sys, tx, ty, tz, sx, sy, sz, sq);
    }
    const DevParts *dpp = gpu_tree ? &dp : nullptr;
    double t1 = now_ms();
    PhaseTimer pt;
    if (rep) {
        rep->ms_setup = t1 - t0;
        rep->ms_total = t1 - t0;
        count_interactions(pl, rep);
        pt.mark("setup: interaction counts (host)");
    }
    if (learned) {
        rc = select_degrees(ctx, *arena, pl, tol, dpp);
        if (rc != BT_OK) {
            bt_plan_free(&pl);
            return rc;
        }
        if (rep) {
            pt.t = now_ms();
            count_learned(pl, rep);
            pt.mark("selection: counts (host)");
            rep->ms_setup = now_ms() - t0;
        }
    }
    SsIn ssin{tq, sw, on_dev};
    rc = run_plan(ctx, *arena, pl, out, on_dev, rep, dpp, shape, nullptr, true, prm.sing == SUBTRACTION ? &ssin : nullptr);
    bt_plan_free(&pl);
    if (rc != BT_OK && !on_dev) memset(out, 0, sizeof(double) * (size_t)nt);
    return rc;
}

// ---------------------------------------------------------------------------
// Sessions: fixed geometry, new charges per evaluation, replayed as a graph
// ---------------------------------------------------------------------------
struct Session {
    int device = 0;
    DeviceCtx *ctx = nullptr;
    Arena tree_arena, arena;        // owned by the session
    DevPlan v;
    bool on_dev = false;
    int ns = 0, nt = 0;
    double *d_qin = nullptr;        // charges in caller order
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[5] = {};
    long long graph_kernels = 0;    // kernel launches per replay
    bt_report base{};               // interaction counts, node counts, setup time
};

void session_free(Session *s)
{
    if (!s) return;
    if (s->ctx) cudaSetDevice(s->device);
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    for (auto &e : s->ev)
        if (e) cudaEventDestroy(e);
    if (s->d_qin) cudaFree(s->d_qin);
    if (s->arena.base) cudaFree(s->arena.base);
    if (s->tree_arena.base) cudaFree(s->tree_arena.base);
    delete s;
}

}  // namespace

extern "C" {

const char *bt_last_error(void) { return g_err; }

long long bt_kernel_launch_count(void) { return g_launches.load(); }

int BaryTreeInterface_ex(int numTargets, int numSources, const double *targetX, const double *targetY,
                         const double *targetZ, const double *targetValue, const double *sourceX,
                         const double *sourceY, const double *sourceZ, const double *sourceValue,
                         const double *sourceWeight, double *outputArray, int kernel, int numKernelParams,
                         const double *kernelParams, int singularity, int approximation, int compute_type,
                         double theta, int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf,
                         double sizeCheck, double beta, int verbosity)
{
    bt_params prm;
    bt_params_setup(&prm, kernel, numKernelParams, kernelParams, singularity, approximation, compute_type, theta,
                    interpOrder, maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, beta, verbosity);
    bt_report rep;
    int rc = eval_common(Systems(numTargets, numSources), targetX, targetY, targetZ, sourceX, sourceY, sourceZ, sourceValue,
                         outputArray, prm, nullptr, verbosity > 0 ? &rep : nullptr, false, targetValue, sourceWeight);
    if (verbosity > 0 && rc == BT_OK) {
        printf("[BaryTree] barytree_b200: %d targets, %d sources, setup %.3f ms, upward %.3f ms, "
               "compute %.3f ms, downward %.3f ms, total %.3f ms\n",
               numTargets, numSources, rep.ms_setup, rep.ms_upward, rep.ms_compute, rep.ms_downward, rep.ms_total);
    }
    return rc;
}

void BaryTreeInterface(int numTargets, int numSources, double *targetX, double *targetY, double *targetZ,
                       double *targetValue, double *sourceX, double *sourceY, double *sourceZ, double *sourceValue,
                       double *sourceWeight, double *outputArray, KERNEL kernel, int numKernelParams,
                       double *kernelParams, SINGULARITY singularity, APPROXIMATION approximation,
                       COMPUTE_TYPE compute_type, double theta, int interpOrder, int maxPerSourceLeaf,
                       int maxPerTargetLeaf, double sizeCheck, double beta, int verbosity)
{
    int rc = BaryTreeInterface_ex(numTargets, numSources, targetX, targetY, targetZ, targetValue, sourceX, sourceY,
                                  sourceZ, sourceValue, sourceWeight, outputArray, kernel, numKernelParams,
                                  kernelParams, singularity, approximation, compute_type, theta, interpOrder,
                                  maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, beta, verbosity);
    if (rc != BT_OK) fprintf(stderr, "[BaryTree] ERROR (%d): %s\n", rc, g_err);
}

int bt_eval(int numTargets, int numSources, const double *targetX, const double *targetY, const double *targetZ,
            const double *sourceX, const double *sourceY, const double *sourceZ, const double *sourceValue,
            double *outputArray, int kernel, double kernelParam, int approximation, int compute_type, double theta,
            int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck, const bt_options *opts,
            bt_report *report)
{
    bt_params prm;
    bt_params_setup(&prm, kernel, 1, &kernelParam, SKIPPING, approximation, compute_type, theta, interpOrder,
                    maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, -1.0, 0);
    return eval_common(Systems(numTargets, numSources), targetX, targetY, targetZ, sourceX, sourceY, sourceZ, sourceValue,
                       outputArray, prm, opts, report);
}

int bt_eval_ex(int numTargets, int numSources, const double *targetX, const double *targetY, const double *targetZ,
               const double *targetValue, const double *sourceX, const double *sourceY, const double *sourceZ,
               const double *sourceValue, const double *sourceWeight, double *outputArray, int kernel,
               int numKernelParams, const double *kernelParams, int singularity, int approximation,
               int compute_type, double theta, int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf,
               double sizeCheck, double beta, const bt_options *opts, bt_report *report)
{
    bt_params prm;
    bt_params_setup(&prm, kernel, numKernelParams, kernelParams, singularity, approximation, compute_type, theta,
                    interpOrder, maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, beta, 0);
    return eval_common(Systems(numTargets, numSources), targetX, targetY, targetZ, sourceX, sourceY, sourceZ, sourceValue,
                       outputArray, prm, opts, report, false, targetValue, sourceWeight);
}

int bt_eval_noalloc(int numTargets, int numSources, const double *targetX, const double *targetY,
                    const double *targetZ, const double *sourceX, const double *sourceY, const double *sourceZ,
                    const double *sourceValue, double *outputArray, int kernel, double kernelParam,
                    int approximation, int compute_type, double theta, int interpOrder, int maxPerSourceLeaf,
                    int maxPerTargetLeaf, double sizeCheck, int precision, int device)
{
    bt_params prm;
    bt_params_setup(&prm, kernel, 1, &kernelParam, SKIPPING, approximation, compute_type, theta, interpOrder,
                    maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, -1.0, 0);
    bt_options opts;
    memset(&opts, 0, sizeof opts);
    opts.precision = precision;
    opts.device = device;
    opts.inputs_on_device = 1;
    return eval_common(Systems(numTargets, numSources), targetX, targetY, targetZ, sourceX, sourceY, sourceZ, sourceValue,
                       outputArray, prm, &opts, nullptr, true);
}

int bt_eval_batch(int numSystems, const long long *targetOffsets, const long long *sourceOffsets,
                  const double *targetX, const double *targetY, const double *targetZ, const double *sourceX,
                  const double *sourceY, const double *sourceZ, const double *sourceValue, double *outputArray,
                  int kernel, double kernelParam, int approximation, int compute_type, double theta,
                  int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck,
                  const bt_options *opts, bt_report *report)
{
    g_err[0] = 0;
    if (numSystems < 1 || !targetOffsets || !sourceOffsets) {
        set_err("a batch needs at least one system and both offset arrays");
        return BT_ERR_PARAM;
    }
    if (targetOffsets[0] != 0 || sourceOffsets[0] != 0) {
        set_err("offsets must start at 0");
        return BT_ERR_PARAM;
    }
    for (int k = 0; k < numSystems; k++)
        if (targetOffsets[k + 1] < targetOffsets[k] || sourceOffsets[k + 1] < sourceOffsets[k]) {
            set_err("offsets must not decrease (system %d)", k);
            return BT_ERR_PARAM;
        }
    bt_params prm;
    bt_params_setup(&prm, kernel, 1, &kernelParam, SKIPPING, approximation, compute_type, theta, interpOrder,
                    maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, -1.0, 0);
    return eval_common(Systems(numSystems, targetOffsets, sourceOffsets), targetX, targetY, targetZ, sourceX, sourceY,
                       sourceZ, sourceValue, outputArray, prm, opts, report);
}

int bt_direct(int numTargets, int numSources, const double *targetX, const double *targetY, const double *targetZ,
              const double *sourceX, const double *sourceY, const double *sourceZ, const double *sourceValue,
              double *outputArray, int kernel, double kernelParam, int device)
{
    return bt_direct_ex(numTargets, numSources, targetX, targetY, targetZ, sourceX, sourceY, sourceZ, sourceValue,
                        outputArray, kernel, 1, &kernelParam, device);
}

int bt_direct_ex(int numTargets, int numSources, const double *targetX, const double *targetY, const double *targetZ,
                 const double *sourceX, const double *sourceY, const double *sourceZ, const double *sourceValue,
                 double *outputArray, int kernel, int numKernelParams, const double *kernelParams, int device)
{
    return bt_direct_full(numTargets, numSources, targetX, targetY, targetZ, nullptr, sourceX, sourceY, sourceZ,
                          sourceValue, nullptr, outputArray, kernel, numKernelParams, kernelParams, SKIPPING, device);
}

int bt_direct_full(int numTargets, int numSources, const double *targetX, const double *targetY,
                   const double *targetZ, const double *targetValue, const double *sourceX, const double *sourceY,
                   const double *sourceZ, const double *sourceValue, const double *sourceWeight, double *outputArray,
                   int kernel, int numKernelParams, const double *kernelParams, int singularity, int device)
{
    g_err[0] = 0;
    if (numTargets < 0 || numSources < 0) { set_err("negative count"); return BT_ERR_PARAM; }
    if (singularity != SKIPPING && singularity != SUBTRACTION) { set_err("invalid singularity"); return BT_ERR_PARAM; }
    if (numTargets == 0) return BT_OK;
    if (!targetX || !targetY || !targetZ || !outputArray || (numSources > 0 && (!sourceX || !sourceY || !sourceZ || !sourceValue))) {
        set_err("NULL array");
        return BT_ERR_PARAM;
    }
    if (kernel != COULOMB && kernel != YUKAWA && kernel != REGULARIZED_COULOMB && kernel != REGULARIZED_YUKAWA &&
        kernel != ATAN && kernel != SIN_OVER_R && kernel != MQ && kernel != RBS_U && kernel != RBS_V && kernel != USER) {
        set_err("kernel not provided");
        return BT_ERR_UNSUPPORTED;
    }
    // The direct sum subtracts only for the kernels that have a subtraction
    // pair term; the others ignore the setting, as the reference's direct
    // driver does (interaction_compute_direct.c:26-231, interaction_compute_correction.c:22-45).
    const bool ss = singularity == SUBTRACTION && bt::ss_direct_kernel(kernel);
    if (ss && (!targetValue || (numSources > 0 && !sourceWeight))) {
        set_err("singularity subtraction needs target charges and source weights");
        return BT_ERR_PARAM;
    }
    if (ss && numKernelParams < (kernel == REGULARIZED_COULOMB || kernel == REGULARIZED_YUKAWA ? 2 : 1)) {
        set_err("kernel needs more parameters");
        return BT_ERR_PARAM;
    }
    const double kernelParam = numKernelParams > 0 && kernelParams ? kernelParams[0] : 0.0;
    const double kernelParam2 = numKernelParams > 1 && kernelParams ? kernelParams[1] : 0.0;
    DeviceCtx *ctx = nullptr;
    int rc = get_ctx(device, &ctx);
    if (rc != BT_OK) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t st = ctx->stream;
    double *d_t[4], *d_s[5], *d_o;
    {
        Layout L;
        for (int i = 0; i < 4; i++) L.add(&d_t[i], numTargets);
        for (int i = 0; i < 5; i++) L.add(&d_s[i], numSources);
        L.add(&d_o, numTargets);
        if (!ctx->arena.reserve(L.total())) { set_err("device allocation failed"); return BT_ERR_CUDA; }
        L.bind(ctx->arena);
        const int ntc = ss ? 4 : 3, nsc = ss ? 5 : 4;
        const double *ht[4] = {targetX, targetY, targetZ, targetValue};
        const double *hs[5] = {sourceX, sourceY, sourceZ, sourceValue, sourceWeight};
        for (int i = 0; i < ntc; i++) CK(cudaMemcpyAsync(d_t[i], ht[i], sizeof(double) * numTargets, cudaMemcpyHostToDevice, st));
        if (numSources > 0)
            for (int i = 0; i < nsc; i++) CK(cudaMemcpyAsync(d_s[i], hs[i], sizeof(double) * numSources, cudaMemcpyHostToDevice, st));
        if (ss) {
            bt::launch_ss_direct(kernel, numTargets, numSources, d_t[0], d_t[1], d_t[2], d_t[3], d_s[0], d_s[1], d_s[2],
                                 d_s[3], d_s[4], kernelParam, kernelParam2, d_o, st);
            bt::launch_ss_correction(numTargets, bt::ss_correction_constant(kernel, kernelParam), d_t[3], d_o, st);
            g_launches += 2;
        } else {
            bt::launch_direct(kernel, numTargets, numSources, d_t[0], d_t[1], d_t[2], d_s[0], d_s[1], d_s[2], d_s[3],
                              kernelParam, d_o, st, kernelParam2);
            g_launches += 1;
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(outputArray, d_o, sizeof(double) * numTargets, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
done:
    return rc;
}

int bt_measure_peaks(int device, double *fp64_tflops, double *fp32_tflops, double *rsqrt_gops)
{
    DeviceCtx *ctx = nullptr;
    int rc = get_ctx(device, &ctx);
    if (rc != BT_OK) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { set_err("device query failed"); return BT_ERR_CUDA; }
    int sms = prop.multiProcessorCount;
    if (!ctx->arena.reserve((size_t)sms * 8 * 256 * sizeof(double))) { set_err("device allocation failed"); return BT_ERR_CUDA; }
    double ops;
    float ms = bt::run_probe(0, sms, &ops, ctx->arena.base, ctx->stream);
    if (fp64_tflops) *fp64_tflops = 2.0 * ops / (ms * 1e-3) / 1e12;
    ms = bt::run_probe(1, sms, &ops, ctx->arena.base, ctx->stream);
    if (fp32_tflops) *fp32_tflops = 2.0 * ops / (ms * 1e-3) / 1e12;
    ms = bt::run_probe(2, sms, &ops, ctx->arena.base, ctx->stream);
    if (rsqrt_gops) *rsqrt_gops = ops / (ms * 1e-3) / 1e9;
    g_launches += 6;
    if (cudaGetLastError() != cudaSuccess) { set_err("probe launch failed"); return BT_ERR_CUDA; }
    return BT_OK;
}

long bt_lists(int numTargets, int numSources, const double *targetX, const double *targetY, const double *targetZ,
              const double *sourceX, const double *sourceY, const double *sourceZ, int compute_type,
              int approximation, double theta, int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf,
              double sizeCheck, int *units, int *nodes, int *entries, long cap)
{
    return bt_lists_ex(numTargets, numSources, targetX, targetY, targetZ, sourceX, sourceY, sourceZ, compute_type,
                       approximation, theta, interpOrder, maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, BT_TREE_HOST,
                       0, units, nodes, entries, cap);
}

long bt_lists_ex(int numTargets, int numSources, const double *targetX, const double *targetY,
                 const double *targetZ, const double *sourceX, const double *sourceY, const double *sourceZ,
                 int compute_type, int approximation, double theta, int interpOrder, int maxPerSourceLeaf,
                 int maxPerTargetLeaf, double sizeCheck, int tree_build, int device, int *units, int *nodes,
                 int *entries, long cap)
{
    g_err[0] = 0;
    if (tree_build != BT_TREE_GPU && tree_build != BT_TREE_HOST) {
        set_err("invalid tree_build %d", tree_build);
        return -2;
    }
    bt_plan pl;
    memset(&pl, 0, sizeof pl);
    bt_params_setup(&pl.prm, COULOMB, 0, nullptr, SKIPPING, approximation, compute_type, theta, interpOrder,
                    maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, -1.0, 0);
    if (tree_build == BT_TREE_HOST) {
        build_plan(pl, numTargets, numSources, targetX, targetY, targetZ, sourceX, sourceY, sourceZ, nullptr);
    } else {
        // the evaluation path's own planning: trees built on the GPU, then the lists
        DeviceCtx *ctx = nullptr;
        if (get_ctx(device, &ctx) != BT_OK) return -2;
        std::lock_guard<std::mutex> lk(ctx->mu);
        DevParts dp;
        int e = build_plan_gpu(ctx, ctx->tree_arena, pl, Systems(numTargets, numSources), targetX, targetY, targetZ,
                               sourceX, sourceY, sourceZ, nullptr, false, dp);
        if (e == BT_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            set_err("CUDA error after the tree build");
            e = BT_ERR_CUDA;
        }
        if (e != BT_OK) {
            bt_plan_free(&pl);
            return -2;
        }
    }
    *units = pl.pp.rows;
    *nodes = compute_type == CLUSTER_PARTICLE ? pl.tt.n : pl.st.n;
    long cnt = 0;
    for (int u = 0; u < pl.pp.rows; u++) {
        const bt_csr *kinds[4] = {&pl.pp, &pl.ap, &pl.pc, &pl.cp};
        for (int k = 0; k < 4; k++)
            for (int64_t e = kinds[k]->off[u]; e < kinds[k]->off[u + 1]; e++) {
                if (cnt < cap) {
                    entries[3 * cnt] = u; entries[3 * cnt + 1] = k; entries[3 * cnt + 2] = kinds[k]->idx[e];
                }
                cnt++;
            }
    }
    bt_plan_free(&pl);
    return cnt <= cap ? cnt : -1;
}

long bt_selector_nweights(void) { return bt::MLP_NWEIGHTS; }

int bt_selector_set(const float *weights, long count)
{
    g_err[0] = 0;
    if (!weights || count != bt::MLP_NWEIGHTS) {
        set_err("selector needs %d weights", bt::MLP_NWEIGHTS);
        return BT_ERR_PARAM;
    }
    std::lock_guard<std::mutex> lk(g_selector_mu);
    g_selector.assign(weights, weights + count);
    return BT_OK;
}

long bt_selector_training_data(int n, const double *x, const double *y, const double *z, const double *q,
                               double theta, int leaf, int nsamples, unsigned seed, float *features, float *labels,
                               int device)
{
    g_err[0] = 0;
    if (n <= 0 || !x || !y || !z || !q || !features || !labels || nsamples <= 0 || leaf < 1) {
        set_err("invalid arguments");
        return -BT_ERR_PARAM;
    }
    DeviceCtx *ctx = nullptr;
    int rc = get_ctx(device, &ctx);
    if (rc != BT_OK) return -rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t st = ctx->stream;
    bt_plan pl;
    memset(&pl, 0, sizeof pl);
    // lists as the fixed-degree-10 method builds them (the size check of the
    // MAC depends on the degree), so training samples the interactions the
    // selector is later asked about
    bt_params_setup(&pl.prm, COULOMB, 0, nullptr, SKIPPING, LAGRANGE, PARTICLE_CLUSTER, theta, 10, leaf, leaf, 1.0,
                    -1.0, 0);
    build_plan(pl, n, n, x, y, z, x, y, z, q);
    const bt_tree &S = pl.st, &T = pl.tt;
    // sample particle-cluster entries of every size (the exact sums run over
    // all of a cluster's particles for up to 32 targets)
    std::vector<int> tn_, sn_;
    {
        std::vector<std::pair<int, int>> all;
        for (int u = 0; u < pl.t_approx.rows; u++)
            for (int64_t k = pl.t_approx.off[u]; k < pl.t_approx.off[u + 1]; k++)
                all.push_back({T.leaves[u], pl.t_approx.idx[k]});
        uint64_t s = seed * 6364136223846793005ULL + 1442695040888963407ULL;
        int want = std::min<int>(nsamples, (int)all.size());
        for (int i = 0; i < want; i++) {        // partial Fisher-Yates with a 64-bit LCG
            s = s * 6364136223846793005ULL + 1442695040888963407ULL;
            size_t j = i + (size_t)((s >> 33) % (all.size() - i));
            std::swap(all[i], all[j]);
            tn_.push_back(all[i].first);
            sn_.push_back(all[i].second);
        }
    }
    const int ns_ = (int)tn_.size();
    std::vector<double> sctr, srad, tctr, trad;
    node_geometry(S, sctr, srad);
    node_geometry(T, tctr, trad);
    std::vector<hvec<double>> grids(bt::MLP_DMAX + 1);
    hvec<double> slen;
    for (int d = bt::MLP_DMIN; d <= bt::MLP_DMAX; d++) fill_grids(S, d, grids[d], slen);
    double *d_sx, *d_sy, *d_sz, *d_sq, *d_tx, *d_ty, *d_tz, *d_mom, *d_sctr, *d_tctr, *d_srad, *d_trad, *d_slen;
    int *d_sibeg, *d_snum, *d_tibeg, *d_tnum, *d_snch, *d_sch, *d_sleaves, *d_slvl, *d_tn, *d_sn;
    float *d_feat, *d_lab;
    double *d_grid[bt::MLP_DMAX + 1] = {}, *d_Q[bt::MLP_DMAX + 1] = {};
    Layout L;
    L.add(&d_sx, n); L.add(&d_sy, n); L.add(&d_sz, n); L.add(&d_sq, n); L.add(&d_tx, n); L.add(&d_ty, n); L.add(&d_tz, n);
    L.add(&d_mom, 2 * (size_t)S.n); L.add(&d_sctr, sctr.size()); L.add(&d_tctr, tctr.size());
    L.add(&d_srad, srad.size()); L.add(&d_trad, trad.size()); L.add(&d_slen, slen.size());
    L.add(&d_sibeg, S.n); L.add(&d_snum, S.n); L.add(&d_tibeg, T.n); L.add(&d_tnum, T.n); L.add(&d_snch, S.n);
    L.add(&d_sch, 8 * (size_t)S.n); L.add(&d_sleaves, S.nleaves); L.add(&d_slvl, S.lvl_off[S.max_depth]);
    L.add(&d_tn, ns_); L.add(&d_sn, ns_); L.add(&d_feat, (size_t)ns_ * bt::MLP_IN); L.add(&d_lab, (size_t)ns_ * bt::MLP_OUT);
    for (int d = bt::MLP_DMIN; d <= bt::MLP_DMAX; d++) {
        L.add(&d_grid[d], grids[d].size());
        L.add(&d_Q[d], (size_t)S.n * (d + 1) * (d + 1) * (d + 1));
    }
    long ret = ns_;
    if (!ctx->arena.reserve(L.total())) {
        set_err("device allocation failed");
        bt_plan_free(&pl);
        return -BT_ERR_CUDA;
    }
    L.bind(ctx->arena);
    {
#define UP(dst, src, cnt) CK(cudaMemcpyAsync(dst, src, sizeof(*(src)) * (size_t)(cnt), cudaMemcpyHostToDevice, st))
        UP(d_sx, pl.src.x, n); UP(d_sy, pl.src.y, n); UP(d_sz, pl.src.z, n); UP(d_sq, pl.src.q, n);
        UP(d_tx, pl.tgt.x, n); UP(d_ty, pl.tgt.y, n); UP(d_tz, pl.tgt.z, n);
        UP(d_sctr, sctr.data(), sctr.size()); UP(d_tctr, tctr.data(), tctr.size());
        UP(d_srad, srad.data(), srad.size()); UP(d_trad, trad.data(), trad.size()); UP(d_slen, slen.data(), slen.size());
        UP(d_sibeg, S.ibeg, S.n); UP(d_snum, S.numpar, S.n); UP(d_tibeg, T.ibeg, T.n); UP(d_tnum, T.numpar, T.n);
        UP(d_snch, S.nchild, S.n); UP(d_sch, S.child, 8 * (size_t)S.n); UP(d_sleaves, S.leaves, S.nleaves);
        UP(d_slvl, S.lvl_nodes, S.lvl_off[S.max_depth]); UP(d_tn, tn_.data(), ns_); UP(d_sn, sn_.data(), ns_);
        for (int d = bt::MLP_DMIN; d <= bt::MLP_DMAX; d++) UP(d_grid[d], grids[d].data(), grids[d].size());
#undef UP
        long long launches = 0;
        for (int d = bt::MLP_DMIN; d <= bt::MLP_DMAX; d++) {
            bt::launch_p2m(d, false, S.nleaves, d_sleaves, S.n, d_sibeg, d_snum, d_grid[d], d_slen, nullptr, d_sx, d_sy,
                           d_sz, d_sq, d_Q[d], st);
            launches++;
            for (int l = S.max_depth - 1; l >= 0; l--) {
                int cnt = S.lvl_off[l + 1] - S.lvl_off[l];
                if (cnt > 0) { bt::launch_m2m(d, cnt, d_slvl + S.lvl_off[l], d_snch, d_sch, d_grid[d], d_Q[d], st); launches++; }
            }
        }
        {
            bt::MomentTree mt{S.n, S.nleaves, S.max_depth, d_sleaves, d_sibeg, d_snum, d_snch, d_sch, d_slvl, S.lvl_off};
            launches += bt::launch_node_moments(mt, d_sq, d_mom, st);
        }
        bt::FeatureArgs fa;
        memset(&fa, 0, sizeof fa);
        fa.t_ctr = d_tctr; fa.s_ctr = d_sctr; fa.t_rad = d_trad; fa.s_rad = d_srad; fa.s_mom = d_mom;
        fa.t_numpar = d_tnum; fa.s_numpar = d_snum;
        bt::launch_features_pairs(fa, ns_, d_tn, d_sn, d_feat, st);
        bt::LabelArgs la;
        memset(&la, 0, sizeof la);
        la.tnodes = d_tn; la.snodes = d_sn; la.t_ibeg = d_tibeg; la.t_numpar = d_tnum; la.s_ibeg = d_sibeg;
        la.s_numpar = d_snum; la.tx = d_tx; la.ty = d_ty; la.tz = d_tz; la.sx = d_sx; la.sy = d_sy; la.sz = d_sz;
        la.sq = d_sq; la.t_ctr = d_tctr; la.s_ctr = d_sctr; la.s_mom = d_mom; la.labels = d_lab;
        for (int d = bt::MLP_DMIN; d <= bt::MLP_DMAX; d++) { la.grid[d] = d_grid[d]; la.Q[d] = d_Q[d]; }
        bt::launch_labels(la, ns_, st);
        launches += 3;
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(features, d_feat, sizeof(float) * (size_t)ns_ * bt::MLP_IN, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(labels, d_lab, sizeof(float) * (size_t)ns_ * bt::MLP_OUT, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        g_launches += launches;
    }
done:
    bt_plan_free(&pl);
    return rc == BT_OK ? ret : -rc;
}

int bt_mlp_loss_grad(const float *weights, const float *features, const float *labels, int n, float *grad_out,
                     float *loss_out, int device)
{
    g_err[0] = 0;
    if (!weights || !features || !labels || n <= 0 || !grad_out) { set_err("invalid arguments"); return BT_ERR_PARAM; }
    DeviceCtx *ctx = nullptr;
    int rc = get_ctx(device, &ctx);
    if (rc != BT_OK) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t st = ctx->stream;
    float *d_w, *d_x, *d_y, *d_act, *d_yh, *d_db, *d_loss, *d_g;
    Layout L;
    L.add(&d_w, bt::MLP_NWEIGHTS); L.add(&d_x, (size_t)n * bt::MLP_IN); L.add(&d_y, (size_t)n * bt::MLP_OUT);
    L.add(&d_act, 3 * (size_t)n * bt::MLP_H); L.add(&d_yh, (size_t)n * bt::MLP_OUT);
    L.add(&d_db, 2 * (size_t)n * bt::MLP_H + (size_t)n * bt::MLP_OUT); L.add(&d_loss, n); L.add(&d_g, bt::MLP_NWEIGHTS);
    if (!ctx->arena.reserve(L.total())) { set_err("device allocation failed"); return BT_ERR_CUDA; }
    L.bind(ctx->arena);
    std::vector<float> lossb(n);
    {
        CK(cudaMemcpyAsync(d_w, weights, sizeof(float) * bt::MLP_NWEIGHTS, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_x, features, sizeof(float) * (size_t)n * bt::MLP_IN, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_y, labels, sizeof(float) * (size_t)n * bt::MLP_OUT, cudaMemcpyHostToDevice, st));
        bt::mlp_forward_backward(d_w, n, d_x, d_y, d_act, d_yh, d_db, d_loss, d_g, st);
        g_launches += 12;
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(grad_out, d_g, sizeof(float) * bt::MLP_NWEIGHTS, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(lossb.data(), d_loss, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (loss_out) {
            double s = 0;
            for (int i = 0; i < n; i++) s += lossb[i];
            *loss_out = (float)(s / n);
        }
    }
done:
    return rc;
}

int bt_mlp_predict(const float *weights, const float *features, long n, float *out, int device)
{
    g_err[0] = 0;
    if (!weights || !features || n <= 0 || !out) { set_err("invalid arguments"); return BT_ERR_PARAM; }
    DeviceCtx *ctx = nullptr;
    int rc = get_ctx(device, &ctx);
    if (rc != BT_OK) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t st = ctx->stream;
    float *d_w, *d_x, *d_yh;
    int *d_mlperr;
    Layout L;
    L.add(&d_w, bt::MLP_NWEIGHTS); L.add(&d_x, (size_t)n * bt::MLP_IN); L.add(&d_yh, (size_t)n * bt::MLP_OUT);
    L.add(&d_mlperr, 1);
    if (!ctx->arena.reserve(L.total())) { set_err("device allocation failed"); return BT_ERR_CUDA; }
    L.bind(ctx->arena);
    {
        CK(cudaMemcpyAsync(d_w, weights, sizeof(float) * bt::MLP_NWEIGHTS, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_x, features, sizeof(float) * (size_t)n * bt::MLP_IN, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(d_mlperr, 0, sizeof(int), st));
        bt::mlp_infer_tc(d_w, n, d_x, d_yh, d_mlperr, st);
        g_launches += 1;
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, d_yh, sizeof(float) * (size_t)n * bt::MLP_OUT, cudaMemcpyDeviceToHost, st));
        int mlperr = 0;
        CK(cudaMemcpyAsync(&mlperr, d_mlperr, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (mlperr) {
            set_err("the MLP's tensor-core kernel timed out waiting for its MMAs");
            rc = BT_ERR_TIMEOUT;
        }
    }
done:
    return rc;
}

int bt_selector_train(const float *features, const float *labels, long n, int epochs, int batch, float lr,
                      unsigned seed, float *weights, float *final_loss, int device)
{
    g_err[0] = 0;
    if (!features || !labels || !weights || n <= 0 || epochs <= 0 || batch <= 0) {
        set_err("invalid arguments");
        return BT_ERR_PARAM;
    }
    if (batch > n) batch = (int)n;
    DeviceCtx *ctx = nullptr;
    int rc = get_ctx(device, &ctx);
    if (rc != BT_OK) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t st = ctx->stream;
    const int NW = bt::MLP_NWEIGHTS;
    float *d_w, *d_m, *d_v, *d_g, *d_X, *d_Y, *d_xb, *d_yb, *d_act, *d_yh, *d_db, *d_loss;
    int *d_rows;
    Layout L;
    L.add(&d_w, NW); L.add(&d_m, NW); L.add(&d_v, NW); L.add(&d_g, NW);
    L.add(&d_X, (size_t)n * bt::MLP_IN); L.add(&d_Y, (size_t)n * bt::MLP_OUT);
    L.add(&d_xb, (size_t)batch * bt::MLP_IN); L.add(&d_yb, (size_t)batch * bt::MLP_OUT);
    L.add(&d_act, 3 * (size_t)batch * bt::MLP_H); L.add(&d_yh, (size_t)batch * bt::MLP_OUT);
    L.add(&d_db, 2 * (size_t)batch * bt::MLP_H + (size_t)batch * bt::MLP_OUT); L.add(&d_loss, batch);
    L.add(&d_rows, n);
    if (!ctx->arena.reserve(L.total())) { set_err("device allocation failed"); return BT_ERR_CUDA; }
    L.bind(ctx->arena);
    std::vector<int> perm(n);
    for (long i = 0; i < n; i++) perm[i] = (int)i;
    uint64_t s = seed * 2862933555777941757ULL + 3037000493ULL;
    std::vector<float> lossb(batch);
    double last = 0;
    long long launches = 0;
    {
        CK(cudaMemcpyAsync(d_w, weights, sizeof(float) * NW, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(d_m, 0, sizeof(float) * NW, st));
        CK(cudaMemsetAsync(d_v, 0, sizeof(float) * NW, st));
        CK(cudaMemcpyAsync(d_X, features, sizeof(float) * (size_t)n * bt::MLP_IN, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_Y, labels, sizeof(float) * (size_t)n * bt::MLP_OUT, cudaMemcpyHostToDevice, st));
        int step = 0;
        const long nbatch = n / batch;
        for (int ep = 0; ep < epochs; ep++) {
            for (long i = n - 1; i > 0; i--) {      // Fisher-Yates with a 64-bit LCG
                s = s * 6364136223846793005ULL + 1442695040888963407ULL;
                long j = (long)((s >> 33) % (uint64_t)(i + 1));
                std::swap(perm[i], perm[j]);
            }
            CK(cudaMemcpyAsync(d_rows, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
            for (long b = 0; b < nbatch; b++) {
                bt::gather_rows(batch, bt::MLP_IN, d_rows + b * batch, d_X, d_xb, st);
                bt::gather_rows(batch, bt::MLP_OUT, d_rows + b * batch, d_Y, d_yb, st);
                bt::mlp_forward_backward(d_w, batch, d_xb, d_yb, d_act, d_yh, d_db, d_loss, d_g, st);
                // the input normalisation is fixed: keep its gradient zero
                bt::mlp_adam(NW - 2 * bt::MLP_IN, d_w + 2 * bt::MLP_IN, d_g + 2 * bt::MLP_IN, d_m + 2 * bt::MLP_IN,
                             d_v + 2 * bt::MLP_IN, lr, ++step, st);
                launches += 15;
            }
            CK(cudaStreamSynchronize(st));
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(lossb.data(), d_loss, sizeof(float) * batch, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(weights, d_w, sizeof(float) * NW, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int i = 0; i < batch; i++) last += lossb[i];
        if (final_loss) *final_loss = (float)(last / batch);
        g_launches += launches;
    }
done:
    return rc;
}

int bt_tree_dump(int n, const double *x, const double *y, const double *z, int maxparnode, int *ints, double *dbl, int cap)
{
    return bt_tree_dump_ex(n, x, y, z, maxparnode, BT_TREE_HOST, 0, ints, dbl, nullptr, cap);
}

int bt_tree_dump_ex(int n, const double *x, const double *y, const double *z, int maxparnode, int tree_build,
                    int device, int *ints, double *dbl, int *order, int cap)
{
    g_err[0] = 0;
    if (n < 0 || maxparnode < 1 || (n > 0 && (!x || !y || !z)) || (tree_build != BT_TREE_GPU && tree_build != BT_TREE_HOST)) {
        set_err("invalid tree arguments");
        return -2;
    }
    bt_parts p;
    memset(&p, 0, sizeof p);
    bt_tree t;
    if (tree_build == BT_TREE_HOST) {
        bt_parts_init(&p, n, x, y, z, nullptr);
        bt_tree_build(&t, &p, maxparnode);
        if (order && n > 0) memcpy(order, p.order, sizeof(int) * (size_t)n);
    } else {
        DeviceCtx *ctx = nullptr;
        if (get_ctx(device, &ctx) != BT_OK) return -2;
        std::lock_guard<std::mutex> lk(ctx->mu);
        cudaStream_t st = ctx->stream;
        double *d_x, *d_y, *d_z;
        int *d_ord;
        unsigned char *d_work;
        const size_t wbytes = bt::gpu_tree_work_bytes(n, maxparnode, false);
        Layout L;
        L.add(&d_x, n); L.add(&d_y, n); L.add(&d_z, n); L.add(&d_ord, n); L.add(&d_work, wbytes);
        if (!ctx->tree_arena.reserve(L.total())) { set_err("device allocation failed"); return -2; }
        L.bind(ctx->tree_arena);
        long long launches = 0;
        int e = bt::gpu_build_tree(n, x, y, z, nullptr, maxparnode, bt::GtArrays{d_x, d_y, d_z, nullptr, d_ord}, d_work,
                                   wbytes, &t, st, &launches);
        if (!e && order && n > 0) e = (int)cudaMemcpyAsync(order, d_ord, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st);
        if (!e) e = (int)cudaStreamSynchronize(st);
        g_launches += launches;
        if (e) {
            set_err("CUDA error %s in the tree build", cudaGetErrorString((cudaError_t)e));
            bt_tree_free(&t);
            return -2;
        }
    }
    int nn = t.n;
    if (nn <= cap) {
        for (int i = 0; i < nn; i++) {
            ints[4 * i] = t.ibeg[i] + 1; ints[4 * i + 1] = t.ibeg[i] + t.numpar[i];
            ints[4 * i + 2] = t.nchild[i]; ints[4 * i + 3] = t.level[i];
            double d[7] = {t.x0[i], t.x1[i], t.y0[i], t.y1[i], t.z0[i], t.z1[i], t.rad[i]};
            memcpy(dbl + 7 * i, d, sizeof d);
        }
    }
    bt_tree_free(&t);
    bt_parts_free(&p);
    return nn <= cap ? nn : -1;
}

int bt_session_create(int numSystems, const long long *targetOffsets, const long long *sourceOffsets,
                      const double *targetX, const double *targetY, const double *targetZ, const double *sourceX,
                      const double *sourceY, const double *sourceZ, const double *sourceValue, int kernel,
                      double kernelParam, int approximation, int compute_type, double theta, int interpOrder,
                      int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck, const bt_options *opts,
                      bt_session **session)
{
    g_err[0] = 0;
    if (!session) { set_err("session pointer is NULL"); return BT_ERR_PARAM; }
    *session = nullptr;
    if (numSystems < 1 || (numSystems > 1 && (!targetOffsets || !sourceOffsets))) {
        set_err("a session needs at least one system (offsets for more than one)");
        return BT_ERR_PARAM;
    }
    std::vector<long long> tdef, sdef;
    if (!targetOffsets || !sourceOffsets) {
        set_err("offsets are required (numSystems+1 entries, from 0)");
        return BT_ERR_PARAM;
    }
    if (targetOffsets[0] != 0 || sourceOffsets[0] != 0) { set_err("offsets must start at 0"); return BT_ERR_PARAM; }
    for (int k = 0; k < numSystems; k++)
        if (targetOffsets[k + 1] < targetOffsets[k] || sourceOffsets[k + 1] < sourceOffsets[k]) {
            set_err("offsets must not decrease (system %d)", k);
            return BT_ERR_PARAM;
        }
    const Systems sys(numSystems, targetOffsets, sourceOffsets);
    const int64_t nt64 = sys.toff[sys.n], ns64 = sys.soff[sys.n];
    if (nt64 > INT_MAX || ns64 > INT_MAX) { set_err("more than 2^31-1 particles"); return BT_ERR_PARAM; }
    const int nt = (int)nt64, ns = (int)ns64;
    if (nt < 1 || ns < 1) { set_err("a session needs at least one target and one source"); return BT_ERR_PARAM; }
    bt_params prm;
    bt_params_setup(&prm, kernel, 1, &kernelParam, SKIPPING, approximation, compute_type, theta, interpOrder,
                    maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, -1.0, 0);
    int rc = validate(nt, ns, targetX, targetY, targetZ, sourceX, sourceY, sourceZ, sourceValue, sourceX, prm);
    if (rc != BT_OK) return rc;
    if (opts && opts->tree_build == BT_TREE_HOST) {
        set_err("sessions build their trees on the GPU");
        return BT_ERR_UNSUPPORTED;
    }
    bool learned = false;
    EvalConfig shape;
    double tol = 1e-6;
    rc = parse_options(opts, prm, learned, tol, shape);
    if (rc != BT_OK) return rc;
    const int device = opts ? opts->device : 0;
    DeviceCtx *ctx = nullptr;
    rc = get_ctx(device, &ctx);
    if (rc != BT_OK) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t st = ctx->stream;
    Session *S = new Session;
    S->device = device;
    S->ctx = ctx;
    S->on_dev = opts && opts->inputs_on_device;
    S->ns = ns;
    S->nt = nt;
    double t0 = now_ms();
    bt_plan pl;
    memset(&pl, 0, sizeof pl);
    pl.prm = prm;
    DevParts dp;
    rc = build_plan_gpu(ctx, S->tree_arena, pl, sys, targetX, targetY, targetZ, sourceX, sourceY, sourceZ, sourceValue,
                        S->on_dev, dp);
    if (rc == BT_OK) {
        count_interactions(pl, &S->base);
        if (learned) {
            rc = select_degrees(ctx, S->arena, pl, tol, &dp);
            if (rc == BT_OK) count_learned(pl, &S->base);
        }
    }
    if (rc == BT_OK)
        rc = run_plan(ctx, S->arena, pl, nullptr, true, nullptr, &dp, shape, &S->v, false);
    const int *sorder = dp.sorder;
    bt_plan_free(&pl);
    if (rc == BT_OK && cudaMalloc(&S->d_qin, sizeof(double) * (size_t)ns) != cudaSuccess) {
        cudaGetLastError();
        set_err("device allocation for the session's charges failed");
        rc = BT_ERR_CUDA;
    }
    for (int i = 0; rc == BT_OK && i < 5; i++)
        if (cudaEventCreate(&S->ev[i]) != cudaSuccess) { set_err("event creation failed"); rc = BT_ERR_CUDA; }
    if (rc == BT_OK) {
        // capture: charges into tree order, then the whole device sequence
        cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            bt::launch_gather(ns, sorder, S->d_qin, (double *)S->v.d_sq, st);
            long long launches = 1;
            int rc2 = issue_plan(S->v, st, S->ev, S->v.d_out, launches, true, &ctx->fk);
            e = cudaStreamEndCapture(st, &S->graph);
            if (rc2 != BT_OK) rc = rc2;
            S->graph_kernels = launches;
        }
        if (rc == BT_OK && e == cudaSuccess) e = cudaGraphInstantiate(&S->exec, S->graph, 0);
        if (rc == BT_OK && e != cudaSuccess) {
            set_err("graph capture failed: %s", cudaGetErrorString(e));
            rc = BT_ERR_CUDA;
        }
    }
    if (rc != BT_OK) {
        cudaGetLastError();
        session_free(S);
        return rc;
    }
    S->base.ms_setup = now_ms() - t0;
    S->base.source_nodes = S->v.S_n;
    S->base.target_nodes = S->v.T_n;
    S->base.kernel_launches = (int)S->graph_kernels;
    *session = reinterpret_cast<bt_session *>(S);
    return BT_OK;
}

int bt_session_eval(bt_session *session, const double *sourceValue, double *outputArray, bt_report *report)
{
    g_err[0] = 0;
    Session *S = reinterpret_cast<Session *>(session);
    if (!S || !sourceValue || !outputArray) { set_err("session, charges and output are required"); return BT_ERR_PARAM; }
    std::lock_guard<std::mutex> lk(S->ctx->mu);
    if (cudaSetDevice(S->device) != cudaSuccess) { set_err("cudaSetDevice failed"); return BT_ERR_CUDA; }
    cudaStream_t st = S->ctx->stream;
    const double t0 = now_ms();
    const cudaMemcpyKind in = S->on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind out = S->on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    cudaError_t e = cudaMemcpyAsync(S->d_qin, sourceValue, sizeof(double) * (size_t)S->ns, in, st);
    if (e == cudaSuccess) e = cudaGraphLaunch(S->exec, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(outputArray, S->v.d_out, sizeof(double) * (size_t)S->nt, out, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_err("session evaluation failed: %s", cudaGetErrorString(e));
        return BT_ERR_CUDA;
    }
    g_launches += S->graph_kernels;
    const int erc = check_device_error(S->v, st);
    if (erc != BT_OK) return erc;
    if (report) {
        *report = S->base;
        float a = 0, b = 0, c = 0, d = 0;
        cudaEventElapsedTime(&a, S->ev[0], S->ev[1]);
        cudaEventElapsedTime(&b, S->ev[1], S->ev[2]);
        cudaEventElapsedTime(&c, S->ev[2], S->ev[3]);
        cudaEventElapsedTime(&d, S->ev[3], S->ev[4]);
        cudaGetLastError();
        report->ms_upward = a;
        report->ms_compute = b + c;
        report->ms_downward = d;
        report->ms_eval_kernel = c;
        report->ms_total = now_ms() - t0;
        report->ms_transfer = report->ms_total - (a + b + c + d);
        report->ms_setup = 0.0;
    }
    return BT_OK;
}

int bt_session_destroy(bt_session *session)
{
    Session *S = reinterpret_cast<Session *>(session);
    if (!S) return BT_OK;
    {
        std::lock_guard<std::mutex> lk(S->ctx->mu);
        session_free(S);
    }
    return BT_OK;
}

int bt_tuning_set(int device, int kernel, int approximation, const bt_tuning *t)
{
    g_err[0] = 0;
    if (!tune_key_ok(device, kernel, approximation)) { set_err("invalid device, kernel or approximation"); return BT_ERR_PARAM; }
    if (t && (!bt::mixed_shape_valid(t->targets_per_thread, t->source_tile) ||
              (t->dispatch != BT_DISPATCH_GRID && t->dispatch != BT_DISPATCH_QUEUE))) {
        set_err("invalid tile shape (%d targets per thread, %d-source tiles, dispatch %d)", t->targets_per_thread,
                t->source_tile, t->dispatch);
        return BT_ERR_PARAM;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_has_tuned[device][kernel][approximation] = t != nullptr;
    if (t) g_tuned[device][kernel][approximation] = *t;
    return BT_OK;
}

int bt_tuning_get(int device, int kernel, int approximation, bt_tuning *t, int *installed)
{
    g_err[0] = 0;
    if (!t || !tune_key_ok(device, kernel, approximation)) { set_err("invalid arguments"); return BT_ERR_PARAM; }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const bool has = g_has_tuned[device][kernel][approximation];
    if (has) {
        *t = g_tuned[device][kernel][approximation];
    } else {
        const EvalConfig d;
        t->targets_per_thread = d.tpt; t->source_tile = d.tile;
        t->dispatch = d.queue ? BT_DISPATCH_QUEUE : BT_DISPATCH_GRID; t->ms = 0.0f;
    }
    if (installed) *installed = has ? 1 : 0;
    return BT_OK;
}

int bt_autotune(int numSystems, const long long *targetOffsets, const long long *sourceOffsets,
                const double *targetX, const double *targetY, const double *targetZ, const double *sourceX,
                const double *sourceY, const double *sourceZ, const double *sourceValue, int kernel,
                double kernelParam, int approximation, int compute_type, double theta, int interpOrder,
                int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck, const bt_options *opts,
                bt_tuning *best, bt_tuning *trials, int maxTrials, int *numTrials)
{
    g_err[0] = 0;
    if (numTrials) *numTrials = 0;
    if (!best) { set_err("best is NULL"); return BT_ERR_PARAM; }
    if (!opts || opts->precision != BT_PRECISION_MIXED) {
        set_err("autotuning covers the mixed-precision particle-output kernel: set BT_PRECISION_MIXED");
        return BT_ERR_UNSUPPORTED;
    }
    if (!tune_key_ok(opts->device, kernel, approximation)) { set_err("invalid device, kernel or approximation"); return BT_ERR_PARAM; }
    // the problem as a session with the given dispatch (the shapes are set per trial below)
    bt_options o = *opts;
    o.dispatch = BT_DISPATCH_GRID;
    bt_session *sess = nullptr;
    int rc = bt_session_create(numSystems, targetOffsets, sourceOffsets, targetX, targetY, targetZ, sourceX, sourceY,
                               sourceZ, sourceValue, kernel, kernelParam, approximation, compute_type, theta,
                               interpOrder, maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, &o, &sess);
    if (rc != BT_OK) return rc;
    Session *S = reinterpret_cast<Session *>(sess);
    // one full evaluation, so every array the kernel reads holds its values
    double *scratch = nullptr;
    std::vector<double> hscratch;
    if (S->on_dev) {
        if (cudaMalloc(&scratch, sizeof(double) * (size_t)S->nt) != cudaSuccess) {
            cudaGetLastError();
            bt_session_destroy(sess);
            set_err("device allocation failed");
            return BT_ERR_CUDA;
        }
    } else {
        hscratch.resize((size_t)S->nt);
        scratch = hscratch.data();
    }
    rc = bt_session_eval(sess, sourceValue, scratch, nullptr);
    if (S->on_dev) cudaFree(scratch);
    if (rc != BT_OK) { bt_session_destroy(sess); return rc; }
    if (!S->v.mixed || S->v.n_ev_items <= 0 || S->v.ss) {
        bt_session_destroy(sess);
        set_err("this problem has no mixed particle-output work to tune");
        return BT_ERR_UNSUPPORTED;
    }
    std::vector<bt_tuning> res;
    {
        std::lock_guard<std::mutex> lk(S->ctx->mu);
        cudaSetDevice(S->device);
        cudaStream_t st = S->ctx->stream;
        // sample: every k-th work item of the cost-sorted list (stays sorted)
        const int nit = S->v.n_ev_items;
        const int want = std::max(8192, nit / 16);
        const int k = std::max(1, nit / want);
        std::vector<int2> items((size_t)nit);
        int2 *d_items = nullptr;
        int *d_counter = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        std::vector<int2> sample;
        if (cudaMemcpy(items.data(), S->v.d_evitems, sizeof(int2) * (size_t)nit, cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = BT_ERR_CUDA;
        } else {
            for (int i = 0; i < nit; i += k) sample.push_back(items[(size_t)i]);
            if (cudaMalloc(&d_items, sizeof(int2) * sample.size()) != cudaSuccess ||
                cudaMalloc(&d_counter, sizeof(int)) != cudaSuccess ||
                cudaMemcpy(d_items, sample.data(), sizeof(int2) * sample.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
                rc = BT_ERR_CUDA;
        }
        const int tpts[3] = {1, 2, 4}, tiles[3] = {512, 1024, 2048}, disp[2] = {BT_DISPATCH_GRID, BT_DISPATCH_QUEUE};
        for (int di = 0; di < 2 && rc == BT_OK; di++)
            for (int ti = 0; ti < 3 && rc == BT_OK; ti++)
                for (int li = 0; li < 3 && rc == BT_OK; li++) {
                    bt::MixedTargetsArgs a = mixed_targets_args(S->v);
                    a.items = d_items;
                    a.nitems = (int)sample.size();
                    a.tpt = tpts[ti];
                    a.tile = tiles[li];
                    a.queue = disp[di] == BT_DISPATCH_QUEUE ? d_counter : nullptr;
                    float bestms = 0.0f;
                    for (int r = 0; r < 3; r++) {      // one warm-up launch, then the faster of two
                        if (a.queue && cudaMemsetAsync(d_counter, 0, sizeof(int), st) != cudaSuccess) { rc = BT_ERR_CUDA; break; }
                        cudaEventRecord(e0, st);
                        bt::launch_eval_targets_mixed(S->v.kernel, a, st);
                        cudaEventRecord(e1, st);
                        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) { rc = BT_ERR_CUDA; break; }
                        g_launches += 1;
                        float ms = 0.0f;
                        cudaEventElapsedTime(&ms, e0, e1);
                        if (r == 1 || (r == 2 && ms < bestms)) bestms = ms;
                    }
                    bt_tuning t;
                    t.targets_per_thread = tpts[ti]; t.source_tile = tiles[li]; t.dispatch = disp[di]; t.ms = bestms;
                    res.push_back(t);
                }
        if (rc != BT_OK) set_err("CUDA error while timing the tile shapes: %s", cudaGetErrorString(cudaGetLastError()));
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (d_items) cudaFree(d_items);
        if (d_counter) cudaFree(d_counter);
        cudaGetLastError();
    }
    bt_session_destroy(sess);
    if (rc != BT_OK) return rc;
    size_t bi = 0;
    for (size_t i = 1; i < res.size(); i++)
        if (res[i].ms < res[bi].ms) bi = i;
    *best = res[bi];
    if (trials)
        for (int i = 0; i < maxTrials && i < (int)res.size(); i++) trials[i] = res[(size_t)i];
    if (numTrials) *numTrials = std::min((int)res.size(), trials ? maxTrials : (int)res.size());
    return bt_tuning_set(opts->device, kernel, approximation, best);
}

}  // extern "C"
