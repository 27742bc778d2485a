/*
 * bt_host.h -- host-side data structures of barytree_b200 (C, no CUDA types).
 *
 * The host builds the trees, batches and MAC interaction lists exactly as the
 * reference does (same node sets, boxes, radii, numbering and list
 * membership), then flattens them into CSR arrays that the CUDA side uploads.
 */
#ifndef BT_HOST_H
#define BT_HOST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BT_MAX_DEGREE 16

/* Particles in tree order.  order[i] = caller index of sorted particle i. */
typedef struct {
    int n;
    double *x, *y, *z, *q;
    int *order;
} bt_parts;

/* Flattened tree (struct Tree, src/tree/struct_tree.h:4-43).  ibeg is 0-based.
 * A forest of independent systems' trees (batched evaluation) is one bt_tree
 * whose systems' nodes are numbered consecutively, each system in pre-order. */
typedef struct {
    int n, cap, max_depth;
    int *ibeg, *numpar, *nchild, *child, *parent, *level;
    double *x0, *x1, *y0, *y1, *z0, *z1, *xm, *ym, *zm, *rad;
    int nleaves;
    int *leaves;          /* DFS order (Tree_Fill_Levels, src/tree/tree.c:122-153)  */
    int *lvl_off;         /* max_depth+1 offsets into lvl_nodes                         */
    int *lvl_nodes;       /* non-leaf nodes grouped by level, DFS order within a level  */
    int nroots;           /* systems                                                    */
    int *roots;           /* per system: its root node, -1 for a system with no particles */
    int *leaf_off;        /* nroots+1 offsets: system k's leaves are leaves[leaf_off[k] ..) */
} bt_tree;

/* Compressed row storage: row r holds idx[off[r] .. off[r+1]). */
typedef struct {
    int rows;
    int64_t *off;
    int *idx;
} bt_csr;

typedef struct {
    int kernel, approx, sing, ctype, degree, P, maxs, maxt;
    double theta, size_check, kp, beta;
    double kp2;             /* kernel_params[1] (epsilon of regularized kernels, delta of atan / MQ) */
    int nkp;                /* number of kernel parameters given */
    int verbosity;
    int precision;          /* 0 = FP64, 1 = mixed (FP32 evaluations, FP64 reductions) */
} bt_params;

/* Everything the device side needs for one evaluation. */
typedef struct {
    bt_params prm;
    bt_parts src, tgt;
    bt_tree st, tt;         /* source tree (PC, CC) / leaves = source batches (CP);
                               target tree (CP, CC) / leaves = target batches (PC)   */
    /* reference-shaped lists, indexed by the reference's "target unit":
       PC: target batch; CP: source batch; CC: target node */
    bt_csr pp, ap, pc, cp;
    /* device-shaped work lists */
    int n_units_t;          /* target units for the particle-output pass (leaves of tt) */
    bt_csr t_approx;        /* per target leaf: source nodes evaluated as clusters (PC)  */
    bt_csr t_direct;        /* per target leaf: source nodes evaluated directly (PP)     */
    bt_csr g_cc;            /* per target node: source clusters for M2L (CC)             */
    bt_csr g_cp;            /* per target node: source nodes evaluated onto the grid (CP) */
    unsigned char *a_deg;   /* per t_approx entry: interpolation degree (NULL: prm.degree) */
    long long sel_hist[14]; /* learned selection: entries per degree, [13] = direct instead */
    int same_tree;          /* the targets are the sources: tt is a copy of st            */
} bt_plan;

/* bt_params.c */
void bt_params_setup(bt_params *o, int kernel, int nkp, const double *kp, int sing, int approx,
                     int ctype, double theta, int degree, int maxs, int maxt, double sc, double beta,
                     int verbosity);

/* bt_tree.c */
void bt_parts_init(bt_parts *p, int n, const double *x, const double *y, const double *z, const double *q);
void bt_parts_free(bt_parts *p);
void bt_tree_build(bt_tree *t, bt_parts *p, int maxparnode);
/* Forest of nsys systems: system k holds particles [sys_off[k], sys_off[k+1]). */
void bt_forest_build(bt_tree *t, bt_parts *p, int nsys, const int64_t *sys_off, int maxparnode);
void bt_tree_free(bt_tree *t);
void bt_tree_copy(bt_tree *dst, const bt_tree *src);
/* Node arrays for n nodes (n, cap set), and the leaf / per-level lists of a
 * tree whose node arrays, max_depth and roots are filled. */
void bt_tree_alloc(bt_tree *t, int n);
void bt_tree_finish(bt_tree *t);
/* The roots array for nsys systems (all -1). */
void bt_tree_set_roots(bt_tree *t, int nsys);

/* bt_lists.c */
void bt_csr_free(bt_csr *c);
void bt_csr_empty(bt_csr *c, int rows);   /* rows empty rows */
void bt_plan_lists(bt_plan *pl);        /* reference-shaped lists and device work lists */
void bt_plan_work_lists(bt_plan *pl);   /* device work lists from pl->ap, pp, pc, cp       */
void bt_plan_free(bt_plan *pl);

/* Chebyshev-2 node placement for one node, in FP64 with the host libm,
 * exactly as src/clusters/clusters.c:857-862. */
void bt_cheb_nodes(int n, double a0, double a1, double *out);

#ifdef __cplusplus
}
#endif
#endif
