/*
 * barytree_b200 -- B200-native barycentric treecode behind BaryTree's C entry point.
 *
 * C ABI only: plain pointers, sizes and enums.  All arrays are caller-owned
 * host memory unless a function says otherwise.  Library: libbarytree_b200.so.
 */
#ifndef BARYTREE_B200_H
#define BARYTREE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; only what this header
 * declares is exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* Enum values are fixed by the reference's public header
 * (src/interface/BaryTreeInterface.h:7-48), so existing callers and their
 * ctypes/Fortran bindings pass the same integers. */
#ifndef H_BARYTREE_TYPES_H
#define H_BARYTREE_TYPES_H
typedef enum KERNEL {
    NO_KERNEL, COULOMB, YUKAWA, REGULARIZED_COULOMB, REGULARIZED_YUKAWA,
    ATAN, TCF, DCF, SIN_OVER_R, MQ, RBS_U, RBS_V, USER
} KERNEL;
typedef enum SINGULARITY { NO_SINGULARITY, SKIPPING, SUBTRACTION } SINGULARITY;
typedef enum APPROXIMATION { NO_APPROX, LAGRANGE, HERMITE } APPROXIMATION;
typedef enum COMPUTE_TYPE { NO_COMPUTE_TYPE, PARTICLE_CLUSTER, CLUSTER_PARTICLE, CLUSTER_CLUSTER } COMPUTE_TYPE;
#endif

/* Status codes returned by the *_ex / bt_* entry points. */
enum {
    BT_OK = 0,
    BT_ERR_PARAM = 1,        /* invalid argument (NULL array, bad size, bad enum) */
    BT_ERR_UNSUPPORTED = 2,  /* valid but not provided (the reference exits here too) */
    BT_ERR_CUDA = 3,         /* CUDA runtime error or allocation failure */
    BT_ERR_TIMEOUT = 4,      /* a bounded device wait expired */
    BT_ERR_NO_DEVICE = 5     /* no usable CUDA device */
};

/* Drop-in replacement for the reference entry point
 * (src/interface/BaryTreeInterface.h:52-59, src/interface/BaryTreeInterface.c:18-62).
 * Same arguments, same meaning: outputArray is zeroed, then receives the
 * potential at each target in the caller's order.  Inputs are not modified.
 * The reference exits the process on invalid or unsupported combinations;
 * this version prints the reason and returns with outputArray zeroed
 * (call BaryTreeInterface_ex to get the status).  No MPI is required. */
void BaryTreeInterface(int numTargets, int numSources,
                       double *targetX, double *targetY, double *targetZ, double *targetValue,
                       double *sourceX, double *sourceY, double *sourceZ, double *sourceValue,
                       double *sourceWeight, double *outputArray,
                       KERNEL kernel, int numKernelParams, double *kernelParams,
                       SINGULARITY singularity, APPROXIMATION approximation, COMPUTE_TYPE compute_type,
                       double theta, int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf,
                       double sizeCheck, double beta, int verbosity);

/* Same as BaryTreeInterface, returning a BT_* status instead of exiting. */
int BaryTreeInterface_ex(int numTargets, int numSources,
                         const double *targetX, const double *targetY, const double *targetZ,
                         const double *targetValue,
                         const double *sourceX, const double *sourceY, const double *sourceZ,
                         const double *sourceValue, const double *sourceWeight, double *outputArray,
                         int kernel, int numKernelParams, const double *kernelParams,
                         int singularity, int approximation, int compute_type,
                         double theta, int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf,
                         double sizeCheck, double beta, int verbosity);

/* ---------------------------------------------------------------------- */
/* Extended interface (no counterpart in the reference).                   */
/* ---------------------------------------------------------------------- */

/* Arithmetic of the interaction kernels. */
enum { BT_PRECISION_FP64 = 0,   /* plain FP64 everywhere (the parity path)            */
       BT_PRECISION_MIXED = 1   /* FP32 kernel evaluations on centre-relative coordinates,
                                   compensated per-target accumulation, FP64 boxes, node
                                   placement, coincidence tests and final reduction      */ };

/* Interpolation degree policy. */
enum { BT_DEGREE_FIXED = 0,     /* every approximation uses interpOrder                 */
       BT_DEGREE_LEARNED = 1    /* per-interaction degree from the loaded selector MLP  */ };

/* Per-call options.  Zero-initialise, then set what you need. */
typedef struct bt_options {
    int precision;        /* BT_PRECISION_*                                          */
    int degree_policy;    /* BT_DEGREE_*                                             */
    double tolerance;     /* target relative L2 error for BT_DEGREE_LEARNED           */
    int device;           /* CUDA device ordinal                                      */
    int inputs_on_device; /* 1: the x,y,z,q pointers passed to bt_eval are device
                             pointers (FP64) and output is a device pointer          */
    int tree_build;       /* BT_TREE_GPU (default) or BT_TREE_HOST: where the trees
                             are built; both give the same trees and particle order  */
    int dispatch;         /* mixed evaluation kernels: BT_DISPATCH_AUTO (default: the
                             autotuned dispatch, else one block per work item),
                             BT_DISPATCH_QUEUE (persistent blocks taking cost-sorted
                             work items from a device counter) or BT_DISPATCH_GRID
                             (one block per work item); results are identical     */
    int upward;           /* mixed Lagrange leaf contractions: BT_UPWARD_AUTO (default:
                             leaf P2M, and the leaf L2P of grid outputs, on the
                             tensor cores in 3xTF32 where (n+1)^2 <= 128) or
                             BT_UPWARD_FP64 (FP64 SIMT, as the FP64 path)            */
    /* Target sharding: with shard_count > 1 the call evaluates shard_index's
     * share of the target leaves (contiguous in tree order, equal estimated
     * cost) and leaves the other potentials 0; the sum of the outputs of all
     * shards is the unsharded result, bit for bit without the symmetric
     * pass.  With it, a pair of near-field leaves belongs to the shard that
     * owns its lower leaf, which also adds the partner's side into targets
     * another shard owns; the sum then agrees with the unsharded result to
     * FP64 rounding (the slice sums are grouped by shard).  Trees, lists and proxies
     * are built in full by every shard; with target grids (cluster-particle,
     * cluster-cluster) a shard evaluates the grids of its leaves and their
     * ancestors only, so the grids of shared ancestors are evaluated by
     * every shard that holds a leaf under them.                            */
    int shard_index;
    int shard_count;
    int symmetry;         /* mixed path, targets = sources (all of a batch's systems),
                             Coulomb, Yukawa or regularized Coulomb, leaves of at most 2048
                             particles: BT_SYMMETRY_AUTO (default)
                             evaluates each pair of near-field leaves that list each
                             other (and can hold no close pair) once for both sides;
                             BT_SYMMETRY_OFF evaluates every direction separately.
                             Results agree to FP32 rounding and are deterministic.  */
} bt_options;

enum { BT_TREE_GPU = 0, BT_TREE_HOST = 1 };
enum { BT_DISPATCH_AUTO = 0, BT_DISPATCH_QUEUE = 1, BT_DISPATCH_GRID = 2 };
enum { BT_UPWARD_AUTO = 0, BT_UPWARD_FP64 = 1 };
enum { BT_SYMMETRY_AUTO = 0, BT_SYMMETRY_OFF = 1 };

/* Per-call report (all optional: pass NULL). */
typedef struct bt_report {
    double ms_total, ms_setup, ms_upward, ms_compute, ms_downward, ms_transfer;
    long long num_pp, num_pc, num_cp, num_cc;                 /* cluster-wise interactions */
    long long pp_ptwise, pc_ptwise, cp_ptwise, cc_ptwise;     /* pointwise, counted as the
                                                                 reference counts them
                                                                 (src/drivers/treedriver.c:467-483,757-793) */
    double ms_eval_kernel;     /* device time of the dominant evaluation kernel */
    long long eval_flops;      /* algorithmic FLOPs of that kernel               */
    int source_nodes, target_nodes, kernel_launches;
    long long selected[14];    /* learned selection: entries per degree (index = degree),
                                  index 13 = entries evaluated directly instead */
    long long sym_ptwise;      /* near-field evaluations (both directions counted) served
                                  by the symmetric pass with one 1/r per pair of them   */
} bt_report;

/* Treecode evaluation with options and a report.  Same meaning of the
 * physical arguments as BaryTreeInterface_ex. */
int bt_eval(int numTargets, int numSources,
            const double *targetX, const double *targetY, const double *targetZ,
            const double *sourceX, const double *sourceY, const double *sourceZ,
            const double *sourceValue, double *outputArray,
            int kernel, double kernelParam, int approximation, int compute_type,
            double theta, int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf,
            double sizeCheck, const bt_options *opts, bt_report *report);

/* BaryTreeInterface_ex with options and a report: every argument of the
 * reference entry point (target charges and source weights for singularity
 * subtraction, all kernel parameters, beta) plus the extended options.
 * opts and report may be NULL (FP64, defaults). */
int bt_eval_ex(int numTargets, int numSources,
               const double *targetX, const double *targetY, const double *targetZ,
               const double *targetValue,
               const double *sourceX, const double *sourceY, const double *sourceZ,
               const double *sourceValue, const double *sourceWeight, double *outputArray,
               int kernel, int numKernelParams, const double *kernelParams,
               int singularity, int approximation, int compute_type,
               double theta, int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf,
               double sizeCheck, double beta, const bt_options *opts, bt_report *report);

/* Batched evaluation of independent systems (no counterpart in the
 * reference, which evaluates one system per call).  System k's targets are
 * entries [targetOffsets[k], targetOffsets[k+1]) of the target arrays and of
 * outputArray, its sources entries [sourceOffsets[k], sourceOffsets[k+1]) of
 * the source arrays (offsets: numSystems+1 host entries, starting at 0).
 * Every system gets its own trees and interaction lists, exactly as a
 * separate bt_eval call would build them, and the same potentials bit for
 * bit; all systems share one upward pass, one evaluation kernel and one
 * downward pass, so many small systems fill the GPU together. */
int bt_eval_batch(int numSystems, const long long *targetOffsets, const long long *sourceOffsets,
                  const double *targetX, const double *targetY, const double *targetZ,
                  const double *sourceX, const double *sourceY, const double *sourceZ,
                  const double *sourceValue, double *outputArray,
                  int kernel, double kernelParam, int approximation, int compute_type,
                  double theta, int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf,
                  double sizeCheck, const bt_options *opts, bt_report *report);

/* Sessions (no counterpart in the reference): fixed geometry, new charges.
 * For a solver that evaluates the same particles many times with changing
 * charges (an iterative method whose matrix-vector product is the
 * treecode), bt_session_create builds the trees and interaction lists,
 * makes the degree selection (BT_DEGREE_LEARNED: with the charges given
 * here), uploads everything and captures the whole device sequence (charges
 * into tree order, upward pass, evaluation kernels, downward pass, reorder)
 * as one CUDA graph; bt_session_eval copies in the new charges, replays the
 * graph and copies out the potentials.  Arguments as bt_eval_batch (one
 * system: offsets {0, numTargets} and {0, numSources}); with
 * opts->inputs_on_device the charges and outputs of bt_session_eval are
 * device pointers too.  A session owns its device memory until
 * bt_session_destroy. */
typedef struct bt_session bt_session;
int bt_session_create(int numSystems, const long long *targetOffsets, const long long *sourceOffsets,
                      const double *targetX, const double *targetY, const double *targetZ,
                      const double *sourceX, const double *sourceY, const double *sourceZ,
                      const double *sourceValue, int kernel, double kernelParam,
                      int approximation, int compute_type, double theta, int interpOrder,
                      int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck,
                      const bt_options *opts, bt_session **session);
int bt_session_eval(bt_session *session, const double *sourceValue, double *outputArray,
                    bt_report *report);
int bt_session_destroy(bt_session *session);

/* Autotuning of the mixed-precision particle-output kernel (no counterpart
 * in the reference).  Its tile shape -- targets per thread (1, 2 or 4, with
 * 256 / targets_per_thread threads per block, so a work item is always 256
 * targets of one leaf), near-field sources per shared-memory tile (512,
 * 1024 or 2048) and dispatch (one block per work item, or persistent blocks
 * on a device work queue) -- is picked by timing every candidate on the
 * caller's own workload.  The chosen shape is installed for (device,
 * kernel, approximation): later evaluations and sessions on that device
 * with BT_DISPATCH_AUTO use it (an explicit dispatch option still wins). */
typedef struct bt_tuning {
    int targets_per_thread;   /* 1, 2 or 4                                         */
    int source_tile;          /* 512, 1024 or 2048                                 */
    int dispatch;             /* BT_DISPATCH_GRID or BT_DISPATCH_QUEUE             */
    float ms;                 /* kernel time on the tuning sample (0: not measured) */
} bt_tuning;

/* Builds the problem as bt_session_create does (same arguments; opts must
 * select BT_PRECISION_MIXED), evaluates it once, then times the
 * particle-output kernel in all 18 shapes on a sample of its work items
 * (every k-th of the cost-sorted list, about a sixteenth of a large
 * problem).  best receives the fastest shape; trials (may be NULL)
 * receives up to maxTrials measured shapes and *numTrials their count. */
int bt_autotune(int numSystems, const long long *targetOffsets, const long long *sourceOffsets,
                const double *targetX, const double *targetY, const double *targetZ,
                const double *sourceX, const double *sourceY, const double *sourceZ,
                const double *sourceValue, int kernel, double kernelParam,
                int approximation, int compute_type, double theta, int interpOrder,
                int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck,
                const bt_options *opts, bt_tuning *best, bt_tuning *trials, int maxTrials,
                int *numTrials);

/* Installs a shape for (device, kernel, approximation), e.g. one saved
 * from an earlier bt_autotune; NULL removes it (defaults: 2 targets per
 * thread, 1024-source tiles, one block per work item). */
int bt_tuning_set(int device, int kernel, int approximation, const bt_tuning *tuning);

/* The shape in use for (device, kernel, approximation): the installed one,
 * or the defaults with ms = 0.  *installed (may be NULL) tells which. */
int bt_tuning_get(int device, int kernel, int approximation, bt_tuning *tuning, int *installed);

/* Allocation-free evaluation (no counterpart in the reference).
 *
 * For callers that must not allocate device memory at call time: code
 * running inside a memory pool or arena that owns the whole device, code
 * whose allocations must be known before it starts (real-time or
 * certification settings), and callers that run while another component has
 * reserved all free memory.  This entry point calls no cudaMalloc, cudaFree
 * or allocating library routine.  All of its device scratch (sorted particle
 * copies, tree arrays, interaction lists, proxy charges, grid potentials)
 * lives in one file-scope static device array of BT_NOALLOC_SCRATCH_BYTES,
 * which every GPU that loads the library holds until the process exits.
 *
 * Arguments are those of bt_eval, except that all seven input arrays and
 * outputArray are DEVICE pointers (FP64) on `device`, and precision is a
 * BT_PRECISION_* value.  The result equals bt_eval with inputs_on_device.
 * A call whose scratch need exceeds the static array returns BT_ERR_PARAM
 * with a message giving both sizes (roughly up to 5e5 particles at degree 8).
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress with that device current); make that first call
 * before any stream capture.  Under CUDA's default lazy module loading the
 * array's memory is taken when the library's module is first used on a
 * device (at the latest by that first call), not when the library is
 * loaded: a caller that reserves all of a device's free memory for itself
 * must make its first call of this function (or of any other library
 * function on that device) before doing so.  Every call on a device shares the one array
 * and leaves the previous call's contents in it; all kernels write their
 * scratch before reading it, so nothing needs to start at zero.  Calls
 * through this library are serialised per device by a lock; work that the
 * caller launches itself and that overlaps a call on the GPU must not touch
 * the array (it is private to the library), and two calls that overlapped on
 * the GPU would race on it. */
#define BT_NOALLOC_SCRATCH_BYTES ((size_t)64 << 20)
int bt_eval_noalloc(int numTargets, int numSources,
                    const double *targetX, const double *targetY, const double *targetZ,
                    const double *sourceX, const double *sourceY, const double *sourceZ,
                    const double *sourceValue, double *outputArray,
                    int kernel, double kernelParam, int approximation, int compute_type,
                    double theta, int interpOrder, int maxPerSourceLeaf, int maxPerTargetLeaf,
                    double sizeCheck, int precision, int device);

/* FP64 direct sum on the GPU (the error reference for large N):
 * out[i] = sum_j q_j K(t_i, s_j) with the reference's skipping rules
 * (src/interaction_compute/interaction_compute_direct.c:26-231). */
int bt_direct(int numTargets, int numSources,
              const double *targetX, const double *targetY, const double *targetZ,
              const double *sourceX, const double *sourceY, const double *sourceZ,
              const double *sourceValue, double *outputArray,
              int kernel, double kernelParam, int device);

/* bt_direct with the kernel parameters as an array (two for regularized
 * Yukawa, atan and MQ), like BaryTreeInterface's numKernelParams /
 * kernelParams; covers every kernel this library provides. */
int bt_direct_ex(int numTargets, int numSources,
                 const double *targetX, const double *targetY, const double *targetZ,
                 const double *sourceX, const double *sourceY, const double *sourceZ,
                 const double *sourceValue, double *outputArray, int kernel,
                 int numKernelParams, const double *kernelParams, int device);

/* FP64 direct sum with every argument of the reference's direct driver
 * (src/drivers/directdriver.c:23-122, interaction_compute_direct.c:26-231):
 * with singularity == SUBTRACTION, Coulomb, Yukawa and their regularized
 * forms use the subtraction pair term and add the correction constant times
 * the target charge (interaction_compute_correction.c:22-45); targetValue
 * and sourceWeight are then required.  Other kernels ignore the setting, as
 * in the reference.  outputArray is overwritten. */
int bt_direct_full(int numTargets, int numSources,
                   const double *targetX, const double *targetY, const double *targetZ,
                   const double *targetValue,
                   const double *sourceX, const double *sourceY, const double *sourceZ,
                   const double *sourceValue, const double *sourceWeight, double *outputArray,
                   int kernel, int numKernelParams, const double *kernelParams,
                   int singularity, int device);

/* Interaction lists as the product builds them, in the canonical triple form
 * (unit, kind, node): kind 0 = PP, 1 = approx (PC / CP / CC), 2 = PC (CC
 * mode), 3 = CP (CC mode).  Mirrors InteractionLists_Make
 * (src/interaction_lists/interaction_lists.c:48-234).  Returns the number of
 * triples, or -1 if `cap` is too small. */
long bt_lists(int numTargets, int numSources,
              const double *targetX, const double *targetY, const double *targetZ,
              const double *sourceX, const double *sourceY, const double *sourceZ,
              int compute_type, int approximation, double theta, int interpOrder,
              int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck,
              int *units, int *nodes, int *entries, long cap);

/* bt_lists with the tree build the lists come from: BT_TREE_HOST, or
 * BT_TREE_GPU on `device` (the evaluation path's own planning: trees built
 * on the GPU, then the MAC traversal).  Returns the number of triples, -1 if
 * `cap` is too small, -2 on other errors (bt_last_error).  No counterpart
 * in the reference beyond InteractionLists_Make itself: it lets the parity
 * tests check the lists the evaluation path uses. */
long bt_lists_ex(int numTargets, int numSources,
                 const double *targetX, const double *targetY, const double *targetZ,
                 const double *sourceX, const double *sourceY, const double *sourceZ,
                 int compute_type, int approximation, double theta, int interpOrder,
                 int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck,
                 int tree_build, int device, int *units, int *nodes, int *entries, long cap);

/* Tree summary, as bto_tree in the oracle: per node (ibeg 1-based, iend,
 * num_children, level) and (x_min,x_max,y_min,y_max,z_min,z_max,radius).
 * Mirrors Tree_Sources_Construct (src/tree/tree.c:19-59). */
int bt_tree_dump(int n, const double *x, const double *y, const double *z, int maxparnode,
            int *ints, double *dbl, int cap);

/* bt_tree_dump with the build location (BT_TREE_HOST / BT_TREE_GPU on
 * `device`, inputs in host memory) and, if order is not NULL, the particle
 * permutation (order[i] = input index of sorted particle i; n entries).
 * Returns the node count, -1 if `cap` is too small, -2 on other errors
 * (bt_last_error).  No counterpart in the reference: it checks that both
 * builds give the reference's tree. */
int bt_tree_dump_ex(int n, const double *x, const double *y, const double *z, int maxparnode,
                    int tree_build, int device, int *ints, double *dbl, int *order, int cap);

/* ---------------------------------------------------------------------- */
/* Learned degree selection (no counterpart in the reference).              */
/* A small MLP (6 -> 64 -> 64 -> 64 -> 11, tanh, FP32) predicts, for each    */
/* particle-cluster interaction, log10 of its normalised error at degrees   */
/* 2..12; bt_eval with BT_DEGREE_LEARNED (mixed precision, particle-cluster,*/
/* Lagrange, Coulomb) then uses the lowest degree predicted to meet the     */
/* tolerance, or direct evaluation where that is cheaper or none does.      */
/* Features: log10 source count, log10 target count, (r_c + r_b)/d, r_c/d,  */
/* r_b/d, ||q||_1 / (||q||_2 sqrt(count)).                                  */
/* Weights (floats): mean[6], std[6], W1[6][64], b1[64], W2[64][64], b2[64],*/
/* W3[64][64], b3[64], W4[64][11], b4[11].                                  */
/* ---------------------------------------------------------------------- */
long bt_selector_nweights(void);
int bt_selector_set(const float *weights, long count);
/* Training data made by the treecode itself: builds the particle-cluster
 * lists of the system (targets = sources), samples `nsamples` interactions
 * and writes their features (6 floats each) and labels (11 floats each:
 * log10 of the RMS error at degree d over up to 32 targets of the batch,
 * divided by ||q_cluster||_2 / distance, against the exact FP64 sum over the
 * cluster's particles).  Returns the number of samples written or -status. */
long bt_selector_training_data(int n, const double *x, const double *y, const double *z, const double *q,
                               double theta, int leaf, int nsamples, unsigned seed,
                               float *features, float *labels, int device);
/* Adam training on the GPU with the library's forward/backward kernels;
 * `weights` holds the initial weights (with the input normalisation) and
 * receives the trained ones. */
int bt_selector_train(const float *features, const float *labels, long n, int epochs, int batch, float lr,
                      unsigned seed, float *weights, float *final_loss, int device);
/* Mean-squared-error loss and its gradient (weight layout) on one batch. */
int bt_mlp_loss_grad(const float *weights, const float *features, const float *labels, int n,
                     float *grad_out, float *loss_out, int device);
/* Predicted log10 errors (11 per row). */
int bt_mlp_predict(const float *weights, const float *features, long n, float *out, int device);

/* Throughput microbenchmarks on `device` (the roofline denominators of the
 * SIMT evaluation kernels): dependent-FMA streams in FP64 and FP32 and a
 * reciprocal-square-root stream, each over all SMs.  Results in TFLOP/s
 * (FMA = 2 FLOP) and Gop/s. */
int bt_measure_peaks(int device, double *fp64_tflops, double *fp32_tflops, double *rsqrt_gops);

/* Last error message of the calling thread ("" if none). */
const char *bt_last_error(void);

/* Number of CUDA kernels this library launched in this process (for checks). */
long long bt_kernel_launch_count(void);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* BARYTREE_B200_H */
