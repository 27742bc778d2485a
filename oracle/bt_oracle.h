/*
 * bt_oracle -- CPU FP64 restatement of the BaryTree treecode (test infrastructure).
 *
 * This library is the parity checker for the barytree_b200 product.  Only the
 * tests, the smoke check and the benchmark's CPU-baseline leg load it; the
 * product never links or calls it.
 *
 * Parity is pinned against the reference built from its own sources
 * (oracle/_ref/libBaryTree_ref.so, see oracle/Makefile) and against the
 * reference's known-answer tests (tests/serial_tests.c).
 */
#ifndef BT_ORACLE_H
#define BT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Enum values follow src/interface/BaryTreeInterface.h:7-48. */
enum { BTO_COULOMB = 1, BTO_YUKAWA = 2, BTO_REGULARIZED_COULOMB = 3 };
enum { BTO_SKIPPING = 1, BTO_SUBTRACTION = 2 };
enum { BTO_LAGRANGE = 1, BTO_HERMITE = 2 };
enum { BTO_PARTICLE_CLUSTER = 1, BTO_CLUSTER_PARTICLE = 2, BTO_CLUSTER_CLUSTER = 3 };

/* FP64 direct sum, restating InteractionCompute_Direct
 * (src/interaction_compute/interaction_compute_direct.c:26-231) with the
 * skipping kernels K_*_PP.  out[i] = sum_j q_j K(t_i, s_j).  OpenMP over targets. */
int bto_direct(int nt, const double *tx, const double *ty, const double *tz,
               int ns, const double *sx, const double *sy, const double *sz, const double *sq,
               int kernel, double kernel_param, double *out);

/* Full treecode, same argument list and meaning as BaryTreeInterface
 * (src/interface/BaryTreeInterface.h:52-59).  Returns 0 on success, a negative
 * code for an unsupported combination (the reference exits there). */
int bto_treecode(int numTargets, int numSources,
                 const double *targetX, const double *targetY, const double *targetZ, const double *targetValue,
                 const double *sourceX, const double *sourceY, const double *sourceZ, const double *sourceValue,
                 const double *sourceWeight, double *outputArray,
                 int kernel, int numKernelParams, const double *kernelParams,
                 int singularity, int approximation, int compute_type,
                 double theta, int interpDegree, int maxPerSourceLeaf, int maxPerTargetLeaf,
                 double sizeCheck, double beta, int verbosity);

/* Interaction lists in a canonical flat form, for bit-exact membership checks.
 * Builds the trees/batches and the lists exactly as the treecode does, then
 * writes, for every target unit u (batch for PC, source batch for CP, target
 * node for CC), the list entries of each kind as source-side node indices:
 *   kinds: 0 = PP (direct), 1 = approx (PC for PC, CP for CP, CC for CC),
 *          2 = PC (CC only), 3 = CP (CC only).
 * Output triples (unit, kind, node) in traversal order into `entries`
 * (capacity `cap` triples).  Returns the number of triples, or -1 if `cap`
 * is too small.  `units` receives the number of target units, `nodes` the
 * number of nodes of the tree the entries index. */
long bto_lists(int numTargets, int numSources,
               const double *targetX, const double *targetY, const double *targetZ,
               const double *sourceX, const double *sourceY, const double *sourceZ,
               int compute_type, int approximation, double theta, int interpDegree,
               int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck,
               int *units, int *nodes, int *entries, long cap);

/* Tree summary for structure checks: per node (ibeg, iend, num_children, level)
 * into `ints` (4 per node) and (x_min,x_max,y_min,y_max,z_min,z_max,radius)
 * into `dbl` (7 per node).  Returns the node count, or -1 if cap too small. */
int bto_tree(int n, const double *x, const double *y, const double *z, int maxparnode,
             int *ints, double *dbl, int cap);

#ifdef __cplusplus
}
#endif
#endif
