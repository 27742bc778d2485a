/*
 * bt_oracle.c -- CPU FP64 restatement of the BaryTree treecode.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load this library, and only as the checker.  The product
 * (barytree_b200) neither links nor calls it.
 *
 * Every routine names the reference file:line it restates (paths relative to
 * the BaryTree project root).  The restatement follows the reference's
 * arithmetic order where that matters for parity (node placement, MAC tests,
 * exact-coincidence handling); loops are plain scalar C.
 *
 * Pinning: tests/test_oracle.py checks this library against the reference's
 * known-answer tests (tests/serial_tests.c) and against the reference itself
 * built from its own sources (oracle/_ref/libBaryTree_ref.so) on seeded
 * inputs: bit-exact interaction lists and potentials to 1e-13 relative.
 */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bt_oracle.h"

/* ------------------------------------------------------------------ */
/* small growable int vector                                           */
/* ------------------------------------------------------------------ */
typedef struct { int n, cap; int *v; } ivec;

static void iv_push(ivec *a, int x)
{
    if (a->n == a->cap) {
        a->cap = a->cap ? a->cap * 2 : 16;
        a->v = (int *)realloc(a->v, sizeof(int) * (size_t)a->cap);
    }
    a->v[a->n++] = x;
}

/* ------------------------------------------------------------------ */
/* particles and tree                                                  */
/* ------------------------------------------------------------------ */
typedef struct {
    int n;
    double *x, *y, *z, *q;
    int *order;             /* original index of each (permuted) particle */
} opart;

typedef struct {
    int n, cap, max_depth;
    int *ibeg, *iend, *numpar, *nchild, *child, *level;   /* ibeg/iend 1-based as the reference */
    double *x0, *x1, *y0, *y1, *z0, *z1, *xm, *ym, *zm, *rad;
    ivec leaves;
    ivec *levels;           /* non-leaf nodes per level (Tree_Fill_Levels, src/tree/tree.c:122-153) */
} otree;

static void op_init(opart *p, int n, const double *x, const double *y, const double *z, const double *q)
{
    p->n = n;
    p->x = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    p->y = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    p->z = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    p->q = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    p->order = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) {
        p->x[i] = x[i]; p->y[i] = y[i]; p->z[i] = z[i];
        p->q[i] = q ? q[i] : 0.0;
        p->order[i] = i;
    }
}

static void op_free(opart *p)
{
    free(p->x); free(p->y); free(p->z); free(p->q); free(p->order);
}

static void ot_grow(otree *t)
{
    if (t->n < t->cap) return;
    int c = t->cap ? t->cap * 2 : 64;
#define G(f, T) t->f = (T *)realloc(t->f, sizeof(T) * (size_t)c)
    G(ibeg, int); G(iend, int); G(numpar, int); G(nchild, int); G(level, int);
    G(x0, double); G(x1, double); G(y0, double); G(y1, double); G(z0, double); G(z1, double);
    G(xm, double); G(ym, double); G(zm, double); G(rad, double);
#undef G
    t->child = (int *)realloc(t->child, sizeof(int) * 8 * (size_t)c);
    t->cap = c;
}

static void ot_free(otree *t)
{
    free(t->ibeg); free(t->iend); free(t->numpar); free(t->nchild); free(t->level); free(t->child);
    free(t->x0); free(t->x1); free(t->y0); free(t->y1); free(t->z0); free(t->z1);
    free(t->xm); free(t->ym); free(t->zm); free(t->rad);
    free(t->leaves.v);
    if (t->levels) {
        for (int l = 0; l < t->max_depth; l++) free(t->levels[l].v);
        free(t->levels);
    }
}

/* Partition of the 1-based range [ibeg, iend] on coordinate array `a`
 * about `val`, with the set semantics of cp_partition/pc_partition
 * (src/tree/partition.c:14-90, 94-175): for a range of two or more entries
 * the left part is {a <= val}; a single entry goes left only if a < val
 * (src/tree/partition.c:75-79); an empty range returns ibeg-1.  The order
 * inside each part is not part of the contract (the tree's node sets,
 * boxes and lists do not depend on it); this version keeps it stable. */
static int partition_axis(opart *p, int axis, int ibeg, int iend, double val, double *tmp, int *itmp)
{
    if (ibeg > iend) return ibeg - 1;
    double *a = axis == 0 ? p->x : axis == 1 ? p->y : p->z;
    if (ibeg == iend) return (a[ibeg - 1] < val) ? ibeg : ibeg - 1;
    int lo = ibeg - 1, n = iend - ibeg + 1;
    int nl = 0;
    for (int i = 0; i < n; i++) if (a[lo + i] <= val) nl++;
    double *arr[4] = {p->x, p->y, p->z, p->q};
    int l = 0, r = nl;
    /* destination index of each entry */
    for (int i = 0; i < n; i++) itmp[i] = (a[lo + i] <= val) ? l++ : r++;
    for (int k = 0; k < 4; k++) {
        for (int i = 0; i < n; i++) tmp[itmp[i]] = arr[k][lo + i];
        memcpy(arr[k] + lo, tmp, sizeof(double) * (size_t)n);
    }
    int *ord = (int *)(tmp);  /* reuse: n ints fit in n doubles */
    for (int i = 0; i < n; i++) ord[itmp[i]] = p->order[lo + i];
    memcpy(p->order + lo, ord, sizeof(int) * (size_t)n);
    return ibeg - 1 + nl;
}

static double omin(const double *a, int n) { double m = a[0]; for (int i = 1; i < n; i++) if (m > a[i]) m = a[i]; return m; }
static double omax(const double *a, int n) { double m = a[0]; for (int i = 1; i < n; i++) if (m < a[i]) m = a[i]; return m; }

/* Child ranges of a node, restating pc_partition_8 (src/tree/partition.c:178-286):
 * an axis is divided iff its extent >= max extent / sqrt(2), reduced to at most
 * 4 or 2 children by the max_num_children rules; x, then y, then z; the children
 * of the k-th divided axis are appended after the existing ones. */
static int split_node(opart *p, int ibeg, int iend, double xl, double yl, double zl,
                      int max_nc, double xm, double ym, double zm, int ind[8][2],
                      double *tmp, int *itmp)
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
    int nc = 1;
    ind[0][0] = ibeg; ind[0][1] = iend;
    int div[3] = {dx, dy, dz};
    double mid[3] = {xm, ym, zm};
    for (int ax = 0; ax < 3; ax++) {
        if (!div[ax]) continue;
        for (int i = 0; i < nc; i++) {
            int m = partition_axis(p, ax, ind[i][0], ind[i][1], mid[ax], tmp, itmp);
            ind[nc + i][0] = m + 1;
            ind[nc + i][1] = ind[i][1];
            ind[i][1] = m;
        }
        nc *= 2;
    }
    return nc;
}

/* Recursive construction, restating TreeLinkedList_Sources_Construct /
 * TreeLinkedList_Targets_Construct (src/tree/tree_linked_list.c:16-280) and the
 * pre-order numbering of TreeLinkedList_SetIndex (:284-293). */
static int build_node(otree *t, opart *p, int ibeg, int iend, int maxpar, int level,
                      double *tmp, int *itmp)
{
    ot_grow(t);
    int idx = t->n++;
    int np = iend - ibeg + 1;
    t->ibeg[idx] = ibeg; t->iend[idx] = iend; t->numpar[idx] = np; t->level[idx] = level;
    t->nchild[idx] = 0;
    if (level + 1 > t->max_depth) t->max_depth = level + 1;
    const double *xs = p->x + ibeg - 1, *ys = p->y + ibeg - 1, *zs = p->z + ibeg - 1;
    double x0 = omin(xs, np), x1 = omax(xs, np);
    double y0 = omin(ys, np), y1 = omax(ys, np);
    double z0 = omin(zs, np), z1 = omax(zs, np);
    double xl = x1 - x0, yl = y1 - y0, zl = z1 - z0;
    t->x0[idx] = x0; t->x1[idx] = x1; t->y0[idx] = y0; t->y1[idx] = y1; t->z0[idx] = z0; t->z1[idx] = z1;
    t->xm[idx] = (x1 + x0) / 2.0; t->ym[idx] = (y1 + y0) / 2.0; t->zm[idx] = (z1 + z0) / 2.0;
    t->rad[idx] = sqrt(xl * xl + yl * yl + zl * zl) / 2.0;
    if (np > maxpar) {
        int max_nc = (np < 2 * maxpar) ? 2 : (np < 4 * maxpar) ? 4 : 8;
        int ind[8][2];
        int nc = split_node(p, ibeg, iend, xl, yl, zl, max_nc, t->xm[idx], t->ym[idx], t->zm[idx],
                            ind, tmp, itmp);
        int kids[8], nk = 0;
        for (int i = 0; i < nc; i++) {
            if (ind[i][0] <= ind[i][1]) {
                int c = build_node(t, p, ind[i][0], ind[i][1], maxpar, level + 1, tmp, itmp);
                kids[nk++] = c;
            }
        }
        t->nchild[idx] = nk;
        for (int i = 0; i < nk; i++) t->child[8 * idx + i] = kids[i];
    }
    return idx;
}

/* Leaves and per-level lists in DFS order (Tree_Fill_Levels, src/tree/tree.c:122-153). */
static void fill_levels(otree *t, int idx, int level)
{
    if (t->nchild[idx] == 0) { iv_push(&t->leaves, idx); return; }
    iv_push(&t->levels[level], idx);
    for (int i = 0; i < t->nchild[idx]; i++) fill_levels(t, t->child[8 * idx + i], level + 1);
}

static void tree_build(otree *t, opart *p, int maxpar)
{
    memset(t, 0, sizeof(*t));
    t->max_depth = 1;
    double *tmp = malloc(sizeof(double) * (size_t)(p->n > 0 ? p->n : 1));
    int *itmp = malloc(sizeof(int) * (size_t)(p->n > 0 ? p->n : 1));
    build_node(t, p, 1, p->n, maxpar, 0, tmp, itmp);
    free(tmp); free(itmp);
    t->levels = calloc((size_t)t->max_depth, sizeof(ivec));
    fill_levels(t, 0, 0);
}

/* ------------------------------------------------------------------ */
/* run parameters                                                      */
/* ------------------------------------------------------------------ */
typedef struct {
    int kernel, approx, sing, ctype, degree, P, maxs, maxt;
    double theta, size_check, kp;
} oparams;

/* RunParams_Setup (src/run_params/run_params.c:13-131), including the
 * beta-driven choice of theta and degree (:51-120, CPU leaf sizes :107-119). */
static void params_setup(oparams *o, int kernel, int nkp, const double *kp, int sing, int approx,
                         int ctype, double theta, int degree, int maxs, int maxt, double sc, double beta)
{
    o->kernel = kernel; o->sing = sing; o->approx = approx; o->ctype = ctype;
    o->kp = (nkp > 0 && kp) ? kp[0] : 0.0;
    if (beta < 0 || beta > 1) {
        o->theta = theta; o->degree = degree; o->size_check = sc; o->maxs = maxs; o->maxt = maxt;
    } else {
        double tmin = 0.55, tmax = 0.95, es, nmin = 1, nmax, et = 3;
        if (ctype == BTO_PARTICLE_CLUSTER || ctype == BTO_CLUSTER_PARTICLE) {
            es = 2;
            if (approx == BTO_LAGRANGE) { o->size_check = 1.0; nmax = 12; }
            else { o->size_check = 4.0; nmax = 9; }
        } else {
            o->size_check = 1.0; es = 1.75; nmax = 12;
        }
        o->theta = tmax - (tmax - tmin) * pow(beta, es);
        o->degree = (int)(nmax - (nmax - nmin) * pow(1. - beta, et));
        if (ctype == BTO_PARTICLE_CLUSTER) { o->maxs = 50; o->maxt = 5; }
        else if (ctype == BTO_CLUSTER_PARTICLE) { o->maxs = 5; o->maxt = 50; }
        else { o->maxs = 50; o->maxt = 50; }
    }
    o->P = (o->degree + 1) * (o->degree + 1) * (o->degree + 1);
}

/* ------------------------------------------------------------------ */
/* interaction lists                                                   */
/* ------------------------------------------------------------------ */
typedef struct { ivec *pp, *ap, *pc, *cp; int units; } olists;

/* pc_compute_interaction_list (src/interaction_lists/interaction_lists.c:464-533). */
static void pc_list(const otree *t, int node, double br, double bx, double by, double bz,
                    const oparams *o, ivec *ap, ivec *pp)
{
    double tx = bx - t->xm[node], ty = by - t->ym[node], tz = bz - t->zm[node];
    double dist = sqrt(tx * tx + ty * ty + tz * tz);
    if (((t->rad[node] + br) < dist * o->theta) && (t->rad[node] != 0.00)
        && (o->size_check * o->P < t->numpar[node])) {
        iv_push(ap, node);
    } else if (t->nchild[node] == 0) {
        iv_push(pp, node);
    } else {
        for (int i = 0; i < t->nchild[node]; i++)
            pc_list(t, t->child[8 * node + i], br, bx, by, bz, o, ap, pp);
    }
}

/* cc_compute_interaction_list (src/interaction_lists/interaction_lists.c:537-748). */
static void cc_list(const otree *S, int s, const otree *T, int t, const oparams *o, olists *L)
{
    int size_check = (int)(o->size_check * o->P);
    double tx = T->xm[t] - S->xm[s], ty = T->ym[t] - S->ym[s], tz = T->zm[t] - S->zm[s];
    double dist = sqrt(tx * tx + ty * ty + tz * tz);
    if ((S->rad[s] + T->rad[t]) < dist * o->theta) {
        if (S->numpar[s] <= size_check && T->numpar[t] <= size_check) iv_push(&L->pp[t], s);
        else if (S->numpar[s] <= size_check) iv_push(&L->cp[t], s);
        else if (T->numpar[t] <= size_check) iv_push(&L->pc[t], s);
        else iv_push(&L->ap[t], s);
    } else {
        if (T->nchild[t] == 0 && S->nchild[s] == 0) {
            iv_push(&L->pp[t], s);
        } else if (S->nchild[s] == 0) {
            for (int i = 0; i < T->nchild[t]; i++) cc_list(S, s, T, T->child[8 * t + i], o, L);
        } else if (T->nchild[t] == 0) {
            for (int i = 0; i < S->nchild[s]; i++) cc_list(S, S->child[8 * s + i], T, t, o, L);
        } else if (S->numpar[s] < T->numpar[t]) {
            for (int i = 0; i < T->nchild[t]; i++) cc_list(S, s, T, T->child[8 * t + i], o, L);
        } else {
            for (int i = 0; i < S->nchild[s]; i++) cc_list(S, S->child[8 * s + i], T, t, o, L);
        }
    }
}

static void lists_alloc(olists *L, int units)
{
    L->units = units;
    L->pp = calloc((size_t)units, sizeof(ivec));
    L->ap = calloc((size_t)units, sizeof(ivec));
    L->pc = calloc((size_t)units, sizeof(ivec));
    L->cp = calloc((size_t)units, sizeof(ivec));
}

static void lists_free(olists *L)
{
    for (int i = 0; i < L->units; i++) { free(L->pp[i].v); free(L->ap[i].v); free(L->pc[i].v); free(L->cp[i].v); }
    free(L->pp); free(L->ap); free(L->pc); free(L->cp);
}

/* InteractionLists_Make (src/interaction_lists/interaction_lists.c:48-234).
 * For PC/CP: `tree` is the traversed tree and `batches` the leaves of the
 * other side's tree (Batches_*_Construct, src/tree/batches.c:25-90, produce
 * exactly the leaves, in DFS order, of a tree built with the same rule). */
static void lists_make(olists *L, const otree *tree, const otree *bt, const oparams *o)
{
    if (o->ctype == BTO_CLUSTER_CLUSTER) {
        lists_alloc(L, bt->n);
        cc_list(tree, 0, bt, 0, o, L);
    } else {
        lists_alloc(L, bt->leaves.n);
        for (int i = 0; i < bt->leaves.n; i++) {
            int b = bt->leaves.v[i];
            pc_list(tree, 0, bt->rad[b], bt->xm[b], bt->ym[b], bt->zm[b], o, &L->ap[i], &L->pp[i]);
        }
    }
}

/* ------------------------------------------------------------------ */
/* interaction kernels (skipping forms)                                */
/* ------------------------------------------------------------------ */
/* K_Coulomb_PP (src/kernels/coulomb/coulomb_pp.c:8-61), K_Yukawa_PP
 * (src/kernels/yukawa/yukawa_pp.c:9-57), K_RegularizedCoulomb_PP
 * (src/kernels/regularized-coulomb/regularized-coulomb_pp.c:9-61). */
static inline double kpp(int kernel, double kp, double dx, double dy, double dz, double q)
{
    if (kernel == BTO_COULOMB) {
        double r2 = dx * dx + dy * dy + dz * dz;
        return (r2 > DBL_MIN) ? q / sqrt(r2) : 0.0;
    } else if (kernel == BTO_YUKAWA) {
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        return (r > DBL_MIN) ? q * exp(-kp * r) / r : 0.0;
    } else {
        double r2 = dx * dx + dy * dy + dz * dz + kp * kp;
        return q / sqrt(r2);
    }
}

/* Lagrange PC/CP/CC kernel value without the skip test: K_*_PC_Lagrange
 * (src/kernels/coulomb/coulomb_pc.c:9-61; yukawa_pc.c:9-56;
 * regularized-coulomb_pc.c:9-61) and K_*_CP_Lagrange (coulomb_cp.c:9-61). */
static inline double kpc(int kernel, double kp, double dx, double dy, double dz, double q)
{
    if (kernel == BTO_COULOMB) {
        double r2 = dx * dx + dy * dy + dz * dz;
        return q / sqrt(r2);
    } else if (kernel == BTO_YUKAWA) {
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        return q * exp(-kp * r) / r;
    } else {
        double r2 = dx * dx + dy * dy + dz * dz + kp * kp;
        return q / sqrt(r2);
    }
}

/* Hermite PC: K_Coulomb_PC_Hermite (src/kernels/coulomb/coulomb_pc.c:66-138),
 * K_Yukawa_PC_Hermite (src/kernels/yukawa/yukawa_pc.c:61-140),
 * K_RegularizedCoulomb_PC_Hermite (src/kernels/regularized-coulomb/regularized-coulomb_pc.c:67-142).
 * q[k*P + j] is moment k at grid point j. */
static inline double kpc_herm(int kernel, double kp, double dx, double dy, double dz, const double *q, int j, int P)
{
    if (kernel == BTO_YUKAWA) {
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        double r2 = r * r, r3 = r2 * r;
        double rinv = 1 / r, r3inv = rinv * rinv * rinv, r5inv = r3inv * rinv * rinv, r7inv = r5inv * rinv * rinv;
        double k2 = kp * kp, k3 = kp * k2;
        return exp(-kp * r) * (rinv * q[j]
            + r3inv * (1 + kp * r) * (q[P + j] * dx + q[2 * P + j] * dy + q[3 * P + j] * dz)
            + r5inv * (3 + 3 * kp * r + k2 * r2) * (q[4 * P + j] * dx * dy + q[5 * P + j] * dy * dz + q[6 * P + j] * dx * dz)
            + r7inv * (15 + 15 * kp * r + 6 * k2 * r2 + k3 * r3) * q[7 * P + j] * dx * dy * dz);
    }
    double r = (kernel == BTO_COULOMB) ? sqrt(dx * dx + dy * dy + dz * dz)
                                       : sqrt(dx * dx + dy * dy + dz * dz + kp * kp);
    double rinv = 1 / r, r3inv = rinv * rinv * rinv, r5inv = r3inv * rinv * rinv, r7inv = r5inv * rinv * rinv;
    return rinv * q[j]
         + r3inv * (q[P + j] * dx + q[2 * P + j] * dy + q[3 * P + j] * dz)
         + 3 * r5inv * (q[4 * P + j] * dx * dy + q[5 * P + j] * dy * dz + q[6 * P + j] * dx * dz)
         + 15 * r7inv * q[7 * P + j] * dx * dy * dz;
}

/* Hermite CP: K_Coulomb_CP_Hermite (src/kernels/coulomb/coulomb_cp.c:66-184) and
 * K_Yukawa_CP_Hermite (src/kernels/yukawa/yukawa_cp.c:68-190); the regularized
 * Coulomb form (src/kernels/regularized-coulomb/regularized-coulomb_cp.c:68-188)
 * adds eps^2 to r^2.  d = source - grid point.  Adds to out[0..7]. */
static inline void kcp_herm(int kernel, double kp, double dx, double dy, double dz, double q, double *out)
{
    double r2 = dx * dx + dy * dy + dz * dz;
    if (kernel == BTO_REGULARIZED_COULOMB) r2 += kp * kp;
    if (kernel == BTO_YUKAWA) {
        double r = sqrt(r2), r3 = r2 * r, r2inv = 1 / r2;
        double rinvq = q / r * exp(-kp * r);
        double r3inv = rinvq * r2inv, r5inv = r3inv * r2inv, r7inv = r5inv * r2inv;
        double k2 = kp * kp, k3 = kp * k2;
        double d1 = r3inv * (1 + kp * r);
        double d2 = r5inv * (3 + 3 * kp * r + k2 * r2);
        double d3 = r7inv * (15 + 15 * kp * r + 6 * k2 * r2 + k3 * r3);
        out[0] += rinvq; out[1] += d1 * dx; out[2] += d1 * dy; out[3] += d1 * dz;
        out[4] += d2 * dx * dy; out[5] += d2 * dy * dz; out[6] += d2 * dx * dz; out[7] += d3 * dx * dy * dz;
    } else {
        double r2inv = 1 / r2, rinvq = q / sqrt(r2);
        double r3inv = rinvq * r2inv, r5inv = r3inv * r2inv, r7inv = r5inv * r2inv;
        r5inv *= 3.0;
        out[0] += rinvq; out[1] += r3inv * dx; out[2] += r3inv * dy; out[3] += r3inv * dz;
        out[4] += r5inv * dx * dy; out[5] += r5inv * dy * dz; out[6] += r5inv * dx * dz;
        out[7] += r7inv * dx * dy * dz * 15.0;
    }
}

/* ------------------------------------------------------------------ */
/* clusters: Chebyshev grids and the upward pass                       */
/* ------------------------------------------------------------------ */
typedef struct { double *x, *y, *z, *q; int P, nq; } oclust;

/* Chebyshev-2 nodes mapped onto a node's box (src/clusters/clusters.c:857-862). */
static void cheb_nodes(int n, double a0, double a1, double *out)
{
    for (int i = 0; i <= n; i++) {
        double tt = cos(i * M_PI / n);
        out[i] = a0 + (tt + 1.0) / 2.0 * (a1 - a0);
    }
}

static void lag_weights(int n, double *w)   /* src/clusters/clusters.c:864-879 */
{
    for (int j = 0; j <= n; j++) {
        double dj = (j == 0 || j == n) ? 0.5 : 1.0;
        w[j] = ((j % 2 == 0) ? 1 : -1) * dj;
    }
}

/* Fill grid coordinates of every node (cp_comp_interp, src/clusters/clusters.c:1840-1908). */
static void clusters_grid(oclust *c, const otree *t, int n, int herm)
{
    int P = (n + 1) * (n + 1) * (n + 1);
    c->P = P;
    c->nq = herm ? 8 : 1;
    c->x = calloc((size_t)t->n * P, sizeof(double));
    c->y = calloc((size_t)t->n * P, sizeof(double));
    c->z = calloc((size_t)t->n * P, sizeof(double));
    c->q = calloc((size_t)t->n * P * c->nq, sizeof(double));
    double nx[32], ny[32], nz[32];
    for (int i = 0; i < t->n; i++) {
        cheb_nodes(n, t->x0[i], t->x1[i], nx);
        cheb_nodes(n, t->y0[i], t->y1[i], ny);
        cheb_nodes(n, t->z0[i], t->z1[i], nz);
        for (int j = 0; j < P; j++) {
            int k1 = j % (n + 1), k2 = (j / (n + 1)) % (n + 1), k3 = j / ((n + 1) * (n + 1));
            c->x[(size_t)i * P + j] = nx[k1];
            c->y[(size_t)i * P + j] = ny[k2];
            c->z[(size_t)i * P + j] = nz[k3];
        }
    }
}

static void clusters_free(oclust *c) { free(c->x); free(c->y); free(c->z); free(c->q); }

/* Barycentric anterpolation of a set of m points (x,y,z,q) onto node `dst`'s
 * grid, accumulating into Q: pc_comp_ms_modifiedF (src/clusters/clusters.c:800-1004),
 * and with a child's grid as the point set, pc_comp_ms_modifiedF_child_to_parent
 * (:379-582).  Exact coincidence |s - node| < DBL_MIN selects that node. */
static void anterp(int n, const double *nx, const double *ny, const double *nz,
                   int m, const double *sx, const double *sy, const double *sz, const double *sq, double *Q)
{
    int P = (n + 1) * (n + 1) * (n + 1);
    double w[32];
    lag_weights(n, w);
    double *F = malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    int *ex = malloc(sizeof(int) * 3 * (size_t)(m > 0 ? m : 1));
    for (int i = 0; i < m; i++) {
        double sumX = 0, sumY = 0, sumZ = 0;
        ex[3 * i] = ex[3 * i + 1] = ex[3 * i + 2] = -1;
        for (int j = 0; j <= n; j++) {
            double cx = sx[i] - nx[j], cy = sy[i] - ny[j], cz = sz[i] - nz[j];
            if (fabs(cx) < DBL_MIN) ex[3 * i] = j;
            if (fabs(cy) < DBL_MIN) ex[3 * i + 1] = j;
            if (fabs(cz) < DBL_MIN) ex[3 * i + 2] = j;
            sumX += w[j] / cx; sumY += w[j] / cy; sumZ += w[j] / cz;
        }
        double den = 1.0;
        if (ex[3 * i] == -1) den *= sumX;
        if (ex[3 * i + 1] == -1) den *= sumY;
        if (ex[3 * i + 2] == -1) den *= sumZ;
        F[i] = sq[i] / den;
    }
    for (int j = 0; j < P; j++) {
        int k1 = j % (n + 1), k2 = (j / (n + 1)) % (n + 1), k3 = j / ((n + 1) * (n + 1));
        double cx = nx[k1], cy = ny[k2], cz = nz[k3];
        double temp = 0.0;
        for (int i = 0; i < m; i++) {
            double num = 1.0;
            if (ex[3 * i] == -1) num *= w[k1] / (sx[i] - cx); else if (ex[3 * i] != k1) num *= 0;
            if (ex[3 * i + 1] == -1) num *= w[k2] / (sy[i] - cy); else if (ex[3 * i + 1] != k2) num *= 0;
            if (ex[3 * i + 2] == -1) num *= w[k3] / (sz[i] - cz); else if (ex[3 * i + 2] != k3) num *= 0;
            temp += num * F[i];
        }
        Q[j] += temp;
    }
    free(F); free(ex);
}

/* Hermite anterpolation of a node's own particles into 8 moment arrays,
 * pc_comp_ms_modifiedF_hermite (src/clusters/clusters.c:1224-1514). */
static void anterp_hermite(int n, double x0, double x1, double y0, double y1, double z0, double z1,
                           int m, const double *sx, const double *sy, const double *sz, const double *sq, double *Q)
{
    int P = (n + 1) * (n + 1) * (n + 1);
    double nx[32], ny[32], nz[32], ww[32], dj[32], wx[32], wy[32], wz[32];
    for (int i = 0; i <= n; i++) {
        double xx = i * M_PI / n;
        double tt = cos(xx);
        ww[i] = -cos(xx) / (2 * sin(xx) * sin(xx));
        nx[i] = x0 + (tt + 1.0) / 2.0 * (x1 - x0);
        ny[i] = y0 + (tt + 1.0) / 2.0 * (y1 - y0);
        nz[i] = z0 + (tt + 1.0) / 2.0 * (z1 - z0);
    }
    ww[0] = 0.25 * (n * n / 3.0 + 1.0 / 6.0);
    ww[n] = -ww[0];
    for (int j = 0; j <= n; j++) {
        dj[j] = 1.0;
        wx[j] = -4.0 * ww[j] / (x1 - x0);
        wy[j] = -4.0 * ww[j] / (y1 - y0);
        wz[j] = -4.0 * ww[j] / (z1 - z0);
    }
    dj[0] = 0.25; dj[n] = 0.25;
    double *F = malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    int *ex = malloc(sizeof(int) * 3 * (size_t)(m > 0 ? m : 1));
    for (int i = 0; i < m; i++) {
        double sX = 0, sY = 0, sZ = 0;
        ex[3 * i] = ex[3 * i + 1] = ex[3 * i + 2] = -1;
        for (int j = 0; j <= n; j++) {
            double dx = sx[i] - nx[j], dy = sy[i] - ny[j], dz = sz[i] - nz[j];
            if (fabs(dx) < DBL_MIN) ex[3 * i] = j;
            if (fabs(dy) < DBL_MIN) ex[3 * i + 1] = j;
            if (fabs(dz) < DBL_MIN) ex[3 * i + 2] = j;
            sX += dj[j] / (dx * dx) + wx[j] / dx;
            sY += dj[j] / (dy * dy) + wy[j] / dy;
            sZ += dj[j] / (dz * dz) + wz[j] / dz;
        }
        double den = 1.0;
        if (ex[3 * i] == -1) den *= sX;
        if (ex[3 * i + 1] == -1) den *= sY;
        if (ex[3 * i + 2] == -1) den *= sZ;
        F[i] = sq[i] / den;
    }
    for (int j = 0; j < P; j++) {
        int k1 = j % (n + 1), k2 = (j / (n + 1)) % (n + 1), k3 = j / ((n + 1) * (n + 1));
        double t[8] = {0};
        for (int i = 0; i < m; i++) {
            double dx = sx[i] - nx[k1], dy = sy[i] - ny[k2], dz = sz[i] - nz[k3];
            double A[3], B[3];
            A[0] = dj[k1] / (dx * dx) + wx[k1] / dx; B[0] = dj[k1] / dx;
            A[1] = dj[k2] / (dy * dy) + wy[k2] / dy; B[1] = dj[k2] / dy;
            A[2] = dj[k3] / (dz * dz) + wz[k3] / dz; B[2] = dj[k3] / dz;
            int kk[3] = {k1, k2, k3};
            /* moment k uses B on axis a iff bit a of mask[k] is set:
             * order q, dx, dy, dz, dxy, dyz, dxz, dxyz (src/clusters/clusters.c:1406-1491) */
            static const int mask[8] = {0, 1, 2, 4, 3, 6, 5, 7};
            double num[8];
            for (int k = 0; k < 8; k++) num[k] = 1.0;
            for (int a = 0; a < 3; a++) {
                int e = ex[3 * i + a];
                for (int k = 0; k < 8; k++) {
                    int useB = (mask[k] >> a) & 1;
                    if (e == -1) num[k] *= useB ? B[a] : A[a];
                    else if (e != kk[a] || useB) num[k] *= 0;
                }
            }
            for (int k = 0; k < 8; k++) t[k] += num[k] * F[i];
        }
        for (int k = 0; k < 8; k++) Q[k * P + j] += t[k];
    }
    free(F); free(ex);
}

/* Clusters_Sources_Construct (src/clusters/clusters.c:50-200), skipping forms. */
static void clusters_sources(oclust *c, const otree *t, const opart *s, const oparams *o)
{
    int n = o->degree, P = o->P;
    clusters_grid(c, t, n, o->approx == BTO_HERMITE);
    double nx[32], ny[32], nz[32];
    if (o->approx == BTO_LAGRANGE) {
        for (int li = 0; li < t->leaves.n; li++) {
            int i = t->leaves.v[li];
            cheb_nodes(n, t->x0[i], t->x1[i], nx);
            cheb_nodes(n, t->y0[i], t->y1[i], ny);
            cheb_nodes(n, t->z0[i], t->z1[i], nz);
            int b = t->ibeg[i] - 1;
            anterp(n, nx, ny, nz, t->numpar[i], s->x + b, s->y + b, s->z + b, s->q + b, c->q + (size_t)i * P);
        }
        for (int level = t->max_depth - 1; level >= 0; level--) {
            for (int k = 0; k < t->levels[level].n; k++) {
                int p = t->levels[level].v[k];
                cheb_nodes(n, t->x0[p], t->x1[p], nx);
                cheb_nodes(n, t->y0[p], t->y1[p], ny);
                cheb_nodes(n, t->z0[p], t->z1[p], nz);
                for (int ci = 0; ci < t->nchild[p]; ci++) {
                    int ch = t->child[8 * p + ci];
                    anterp(n, nx, ny, nz, P, c->x + (size_t)ch * P, c->y + (size_t)ch * P, c->z + (size_t)ch * P,
                           c->q + (size_t)ch * P, c->q + (size_t)p * P);
                }
            }
        }
    } else {
        for (int i = 0; i < t->n; i++) {
            int b = t->ibeg[i] - 1;
            anterp_hermite(n, t->x0[i], t->x1[i], t->y0[i], t->y1[i], t->z0[i], t->z1[i], t->numpar[i],
                           s->x + b, s->y + b, s->z + b, s->q + b, c->q + (size_t)i * 8 * P);
        }
    }
}

/* ------------------------------------------------------------------ */
/* downward pass                                                       */
/* ------------------------------------------------------------------ */
/* Lagrange interpolation of node grid values Q (nodes nx,ny,nz) at m points,
 * adding to out: cp_comp_pot (src/interaction_compute/interaction_compute_downpass.c:326-497)
 * and, with a child's grid as the points, cp_comp_pot_parent_to_child (:151-323). */
static void interp_lag(int n, const double *nx, const double *ny, const double *nz, const double *Q,
                       int m, const double *tx, const double *ty, const double *tz, double *out)
{
    int P = (n + 1) * (n + 1) * (n + 1);
    double w[32];
    lag_weights(n, w);
    for (int i = 0; i < m; i++) {
        double sumX = 0, sumY = 0, sumZ = 0;
        int eix = -1, eiy = -1, eiz = -1;
        for (int j = 0; j <= n; j++) {
            double cx = tx[i] - nx[j], cy = ty[i] - ny[j], cz = tz[i] - nz[j];
            if (fabs(cx) < DBL_MIN) eix = j;
            if (fabs(cy) < DBL_MIN) eiy = j;
            if (fabs(cz) < DBL_MIN) eiz = j;
            sumX += w[j] / cx; sumY += w[j] / cy; sumZ += w[j] / cz;
        }
        double den = 1.0;
        if (eix == -1) den /= sumX;
        if (eiy == -1) den /= sumY;
        if (eiz == -1) den /= sumZ;
        double temp = 0.0;
        for (int j = 0; j < P; j++) {
            int k1 = j % (n + 1), k2 = (j / (n + 1)) % (n + 1), k3 = j / ((n + 1) * (n + 1));
            double num = 1.0;
            if (eix == -1) num *= w[k1] / (tx[i] - nx[k1]); else if (eix != k1) num *= 0;
            if (eiy == -1) num *= w[k2] / (ty[i] - ny[k2]); else if (eiy != k2) num *= 0;
            if (eiz == -1) num *= w[k3] / (tz[i] - nz[k3]); else if (eiz != k3) num *= 0;
            temp += num * den * Q[j];
        }
        out[i] += temp;
    }
}

/* Hermite interpolation of a node's 8 grid arrays at its targets,
 * cp_comp_pot_hermite (src/interaction_compute/interaction_compute_downpass.c:860-1109). */
static void interp_hermite(int n, double x0, double x1, double y0, double y1, double z0, double z1,
                           const double *Q, int m, const double *tx, const double *ty, const double *tz, double *out)
{
    int P = (n + 1) * (n + 1) * (n + 1);
    double nx[32], ny[32], nz[32], ww[32], dj[32], wx[32], wy[32], wz[32];
    for (int i = 0; i <= n; i++) {
        double xx = i * M_PI / n;
        double tt = cos(xx);
        ww[i] = -cos(xx) / (2 * sin(xx) * sin(xx));
        nx[i] = x0 + (tt + 1.0) / 2.0 * (x1 - x0);
        ny[i] = y0 + (tt + 1.0) / 2.0 * (y1 - y0);
        nz[i] = z0 + (tt + 1.0) / 2.0 * (z1 - z0);
    }
    ww[0] = 0.25 * (n * n / 3.0 + 1.0 / 6.0);
    ww[n] = -ww[0];
    for (int j = 0; j <= n; j++) {
        dj[j] = 1.0;
        wx[j] = -4.0 * ww[j] / (x1 - x0);
        wy[j] = -4.0 * ww[j] / (y1 - y0);
        wz[j] = -4.0 * ww[j] / (z1 - z0);
    }
    dj[0] = 0.25; dj[n] = 0.25;
    static const int mask[8] = {0, 1, 2, 4, 3, 6, 5, 7};
    for (int i = 0; i < m; i++) {
        double sX = 0, sY = 0, sZ = 0;
        int e[3] = {-1, -1, -1};
        for (int j = 0; j <= n; j++) {
            double cx = tx[i] - nx[j], cy = ty[i] - ny[j], cz = tz[i] - nz[j];
            if (fabs(cx) < DBL_MIN) e[0] = j;
            if (fabs(cy) < DBL_MIN) e[1] = j;
            if (fabs(cz) < DBL_MIN) e[2] = j;
            sX += dj[j] / (cx * cx) + wx[j] / cx;
            sY += dj[j] / (cy * cy) + wy[j] / cy;
            sZ += dj[j] / (cz * cz) + wz[j] / cz;
        }
        double den = 1.0;
        if (e[0] == -1) den /= sX;
        if (e[1] == -1) den /= sY;
        if (e[2] == -1) den /= sZ;
        double temp = 0.0;
        for (int j = 0; j < P; j++) {
            int kk[3] = {j % (n + 1), (j / (n + 1)) % (n + 1), j / ((n + 1) * (n + 1))};
            double d[3] = {tx[i] - nx[kk[0]], ty[i] - ny[kk[1]], tz[i] - nz[kk[2]]};
            double A[3], B[3];
            const double *wa[3] = {wx, wy, wz};
            for (int a = 0; a < 3; a++) {
                A[a] = dj[kk[a]] / (d[a] * d[a]) + wa[a][kk[a]] / d[a];
                B[a] = dj[kk[a]] / d[a];
            }
            double num[8];
            for (int k = 0; k < 8; k++) num[k] = 1.0;
            for (int a = 0; a < 3; a++) {
                for (int k = 0; k < 8; k++) {
                    int useB = (mask[k] >> a) & 1;
                    if (e[a] == -1) num[k] *= useB ? B[a] : A[a];
                    else if (e[a] != kk[a] || useB) num[k] *= 0;
                }
            }
            double s = 0;
            for (int k = 0; k < 8; k++) s += num[k] * Q[k * P + j];
            temp += den * s;
        }
        out[i] += temp;
    }
}

/* InteractionCompute_Downpass (src/interaction_compute/interaction_compute_downpass.c:37-142). */
static void downpass(const otree *t, const opart *tg, oclust *c, const oparams *o, double *pot)
{
    int n = o->degree, P = o->P;
    double nx[32], ny[32], nz[32];
    if (o->approx == BTO_LAGRANGE) {
        for (int level = 0; level < t->max_depth; level++) {
            for (int k = 0; k < t->levels[level].n; k++) {
                int p = t->levels[level].v[k];
                cheb_nodes(n, t->x0[p], t->x1[p], nx);
                cheb_nodes(n, t->y0[p], t->y1[p], ny);
                cheb_nodes(n, t->z0[p], t->z1[p], nz);
                for (int ci = 0; ci < t->nchild[p]; ci++) {
                    int ch = t->child[8 * p + ci];
                    interp_lag(n, nx, ny, nz, c->q + (size_t)p * P, P, c->x + (size_t)ch * P,
                               c->y + (size_t)ch * P, c->z + (size_t)ch * P, c->q + (size_t)ch * P);
                }
            }
        }
        for (int li = 0; li < t->leaves.n; li++) {
            int i = t->leaves.v[li];
            cheb_nodes(n, t->x0[i], t->x1[i], nx);
            cheb_nodes(n, t->y0[i], t->y1[i], ny);
            cheb_nodes(n, t->z0[i], t->z1[i], nz);
            int b = t->ibeg[i] - 1;
            interp_lag(n, nx, ny, nz, c->q + (size_t)i * P, t->numpar[i], tg->x + b, tg->y + b, tg->z + b, pot + b);
        }
    } else {
        for (int i = 0; i < t->n; i++) {
            int b = t->ibeg[i] - 1;
            interp_hermite(n, t->x0[i], t->x1[i], t->y0[i], t->y1[i], t->z0[i], t->z1[i],
                           c->q + (size_t)i * 8 * P, t->numpar[i], tg->x + b, tg->y + b, tg->z + b, pot + b);
        }
    }
}

/* ------------------------------------------------------------------ */
/* compute phases                                                      */
/* ------------------------------------------------------------------ */
static void add_pp(const oparams *o, int nt, const double *tx, const double *ty, const double *tz,
                   int ns, const double *sx, const double *sy, const double *sz, const double *sq, double *pot)
{
    for (int i = 0; i < nt; i++) {
        double acc = 0.0;
        for (int j = 0; j < ns; j++) acc += kpp(o->kernel, o->kp, tx[i] - sx[j], ty[i] - sy[j], tz[i] - sz[j], sq[j]);
        pot[i] += acc;
    }
}

static void add_pc(const oparams *o, int nt, const double *tx, const double *ty, const double *tz,
                   const oclust *c, int node, double *pot)
{
    int P = c->P;
    const double *cx = c->x + (size_t)node * P, *cy = c->y + (size_t)node * P, *cz = c->z + (size_t)node * P;
    for (int i = 0; i < nt; i++) {
        double acc = 0.0;
        if (o->approx == BTO_LAGRANGE) {
            const double *q = c->q + (size_t)node * P;
            for (int j = 0; j < P; j++) acc += kpc(o->kernel, o->kp, tx[i] - cx[j], ty[i] - cy[j], tz[i] - cz[j], q[j]);
        } else {
            const double *q = c->q + (size_t)node * 8 * P;
            for (int j = 0; j < P; j++) acc += kpc_herm(o->kernel, o->kp, tx[i] - cx[j], ty[i] - cy[j], tz[i] - cz[j], q, j, P);
        }
        pot[i] += acc;
    }
}

/* Potential at a target node's grid from m points (CP and, for grid points, CC/M2L). */
static void add_cp(const oparams *o, oclust *tc, int tnode, int m, const double *sx, const double *sy,
                   const double *sz, const double *sq)
{
    int P = tc->P;
    const double *cx = tc->x + (size_t)tnode * P, *cy = tc->y + (size_t)tnode * P, *cz = tc->z + (size_t)tnode * P;
    if (o->approx == BTO_LAGRANGE) {
        double *q = tc->q + (size_t)tnode * P;
        for (int i = 0; i < P; i++) {
            double acc = 0.0;
            for (int j = 0; j < m; j++) acc += kpc(o->kernel, o->kp, cx[i] - sx[j], cy[i] - sy[j], cz[i] - sz[j], sq[j]);
            q[i] += acc;
        }
    } else {
        double *q = tc->q + (size_t)tnode * 8 * P;
        for (int i = 0; i < P; i++) {
            double acc[8] = {0};
            for (int j = 0; j < m; j++) kcp_herm(o->kernel, o->kp, sx[j] - cx[i], sy[j] - cy[i], sz[j] - cz[i], sq[j], acc);
            for (int k = 0; k < 8; k++) q[k * P + i] += acc[k];
        }
    }
}

/* ------------------------------------------------------------------ */
/* public entry points                                                 */
/* ------------------------------------------------------------------ */
int bto_direct(int nt, const double *tx, const double *ty, const double *tz,
               int ns, const double *sx, const double *sy, const double *sz, const double *sq,
               int kernel, double kernel_param, double *out)
{
    oparams o; memset(&o, 0, sizeof o);
    o.kernel = kernel; o.kp = kernel_param;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nt; i++) {
        double acc = 0.0;
        for (int j = 0; j < ns; j++) acc += kpp(kernel, kernel_param, tx[i] - sx[j], ty[i] - sy[j], tz[i] - sz[j], sq[j]);
        out[i] = acc;
    }
    return 0;
}

int bto_tree(int n, const double *x, const double *y, const double *z, int maxparnode,
             int *ints, double *dbl, int cap)
{
    opart p; op_init(&p, n, x, y, z, NULL);
    otree t; tree_build(&t, &p, maxparnode);
    int nn = t.n;
    if (nn <= cap) {
        for (int i = 0; i < nn; i++) {
            ints[4 * i] = t.ibeg[i]; ints[4 * i + 1] = t.iend[i]; ints[4 * i + 2] = t.nchild[i]; ints[4 * i + 3] = t.level[i];
            double d[7] = {t.x0[i], t.x1[i], t.y0[i], t.y1[i], t.z0[i], t.z1[i], t.rad[i]};
            memcpy(dbl + 7 * i, d, sizeof d);
        }
    }
    ot_free(&t); op_free(&p);
    return nn <= cap ? nn : -1;
}

static int validate(int nt, int ns, int kernel, int sing, int approx, int ctype, int degree, int maxs, int maxt)
{
    if (nt < 0 || ns < 0) return -1;
    if (kernel < BTO_COULOMB || kernel > BTO_REGULARIZED_COULOMB) return -2;
    if (sing != BTO_SKIPPING) return -2;    /* subtraction forms are not restated here */
    if (approx != BTO_LAGRANGE && approx != BTO_HERMITE) return -2;
    if (ctype < BTO_PARTICLE_CLUSTER || ctype > BTO_CLUSTER_CLUSTER) return -2;
    if (degree < 1 || degree > 30 || maxs < 1 || maxt < 1) return -1;
    return 0;
}

int bto_treecode(int numTargets, int numSources,
                 const double *targetX, const double *targetY, const double *targetZ, const double *targetValue,
                 const double *sourceX, const double *sourceY, const double *sourceZ, const double *sourceValue,
                 const double *sourceWeight, double *outputArray,
                 int kernel, int numKernelParams, const double *kernelParams,
                 int singularity, int approximation, int compute_type,
                 double theta, int interpDegree, int maxPerSourceLeaf, int maxPerTargetLeaf,
                 double sizeCheck, double beta, int verbosity)
{
    (void)targetValue; (void)sourceWeight; (void)verbosity;
    oparams o;
    params_setup(&o, kernel, numKernelParams, kernelParams, singularity, approximation, compute_type,
                 theta, interpDegree, maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, beta);
    int rc = validate(numTargets, numSources, kernel, singularity, approximation, compute_type, o.degree, o.maxs, o.maxt);
    if (rc) return rc;
    if (compute_type == BTO_CLUSTER_CLUSTER && approximation == BTO_HERMITE) return -2;
    memset(outputArray, 0, sizeof(double) * (size_t)numTargets);   /* src/interface/BaryTreeInterface.c:29 */
    if (numTargets == 0 || numSources == 0) return 0;

    opart S, T;
    op_init(&S, numSources, sourceX, sourceY, sourceZ, sourceValue);
    op_init(&T, numTargets, targetX, targetY, targetZ, NULL);
    double *pot = calloc((size_t)numTargets, sizeof(double));
    otree st, tt;
    olists L;
    oclust sc, tc;
    memset(&st, 0, sizeof st); memset(&tt, 0, sizeof tt);
    memset(&sc, 0, sizeof sc); memset(&tc, 0, sizeof tc);

    if (compute_type == BTO_PARTICLE_CLUSTER) {
        /* treedriver PC branch, src/drivers/treedriver.c:350-627 */
        tree_build(&st, &S, o.maxs);
        tree_build(&tt, &T, o.maxt);      /* batches = leaves (src/tree/batches.c:59-90) */
        clusters_sources(&sc, &st, &S, &o);
        lists_make(&L, &st, &tt, &o);
        for (int i = 0; i < tt.leaves.n; i++) {
            int b = tt.leaves.v[i], tb = tt.ibeg[b] - 1, nb = tt.numpar[b];
            for (int k = 0; k < L.ap[i].n; k++)
                add_pc(&o, nb, T.x + tb, T.y + tb, T.z + tb, &sc, L.ap[i].v[k], pot + tb);
            for (int k = 0; k < L.pp[i].n; k++) {
                int s = L.pp[i].v[k], sb = st.ibeg[s] - 1;
                add_pp(&o, nb, T.x + tb, T.y + tb, T.z + tb, st.numpar[s], S.x + sb, S.y + sb, S.z + sb, S.q + sb, pot + tb);
            }
        }
    } else if (compute_type == BTO_CLUSTER_PARTICLE) {
        /* treedriver CP branch, src/drivers/treedriver.c:114-339 */
        tree_build(&tt, &T, o.maxt);
        tree_build(&st, &S, o.maxs);      /* source batches = leaves */
        clusters_grid(&tc, &tt, o.degree, o.approx == BTO_HERMITE);
        lists_make(&L, &tt, &st, &o);
        for (int i = 0; i < st.leaves.n; i++) {
            int b = st.leaves.v[i], sb = st.ibeg[b] - 1, nb = st.numpar[b];
            for (int k = 0; k < L.ap[i].n; k++)
                add_cp(&o, &tc, L.ap[i].v[k], nb, S.x + sb, S.y + sb, S.z + sb, S.q + sb);
            for (int k = 0; k < L.pp[i].n; k++) {
                int t = L.pp[i].v[k], tb = tt.ibeg[t] - 1;
                add_pp(&o, tt.numpar[t], T.x + tb, T.y + tb, T.z + tb, nb, S.x + sb, S.y + sb, S.z + sb, S.q + sb, pot + tb);
            }
        }
        downpass(&tt, &T, &tc, &o, pot);
    } else {
        /* treedriver CC branch, src/drivers/treedriver.c:638-966 */
        tree_build(&st, &S, o.maxs);
        tree_build(&tt, &T, o.maxt);
        clusters_sources(&sc, &st, &S, &o);
        clusters_grid(&tc, &tt, o.degree, 0);
        lists_make(&L, &st, &tt, &o);
        int P = o.P;
        for (int i = 0; i < tt.n; i++) {
            int tb = tt.ibeg[i] - 1, nb = tt.numpar[i];
            for (int k = 0; k < L.ap[i].n; k++) {       /* CC: K_*_CP_Lagrange on grids (interaction_compute_cc.c:121-127) */
                int s = L.ap[i].v[k];
                add_cp(&o, &tc, i, P, sc.x + (size_t)s * P, sc.y + (size_t)s * P, sc.z + (size_t)s * P, sc.q + (size_t)s * P);
            }
            for (int k = 0; k < L.pc[i].n; k++)
                add_pc(&o, nb, T.x + tb, T.y + tb, T.z + tb, &sc, L.pc[i].v[k], pot + tb);
            for (int k = 0; k < L.cp[i].n; k++) {
                int s = L.cp[i].v[k], sb = st.ibeg[s] - 1;
                add_cp(&o, &tc, i, st.numpar[s], S.x + sb, S.y + sb, S.z + sb, S.q + sb);
            }
            for (int k = 0; k < L.pp[i].n; k++) {
                int s = L.pp[i].v[k], sb = st.ibeg[s] - 1;
                add_pp(&o, nb, T.x + tb, T.y + tb, T.z + tb, st.numpar[s], S.x + sb, S.y + sb, S.z + sb, S.q + sb, pot + tb);
            }
        }
        downpass(&tt, &T, &tc, &o, pot);
    }
    /* Particles_Targets_Reorder (src/particles/particles.c:58-94) */
    for (int i = 0; i < numTargets; i++) outputArray[T.order[i]] = pot[i];

    lists_free(&L);
    clusters_free(&sc); clusters_free(&tc);
    ot_free(&st); ot_free(&tt);
    op_free(&S); op_free(&T);
    free(pot);
    return 0;
}

long bto_lists(int numTargets, int numSources,
               const double *targetX, const double *targetY, const double *targetZ,
               const double *sourceX, const double *sourceY, const double *sourceZ,
               int compute_type, int approximation, double theta, int interpDegree,
               int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck,
               int *units, int *nodes, int *entries, long cap)
{
    oparams o;
    params_setup(&o, BTO_COULOMB, 0, NULL, BTO_SKIPPING, approximation, compute_type, theta, interpDegree,
                 maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, -1.0);
    opart S, T;
    op_init(&S, numSources, sourceX, sourceY, sourceZ, NULL);
    op_init(&T, numTargets, targetX, targetY, targetZ, NULL);
    otree st, tt;
    olists L;
    const otree *trav;
    if (compute_type == BTO_CLUSTER_PARTICLE) {
        tree_build(&tt, &T, o.maxt);
        tree_build(&st, &S, o.maxs);
        lists_make(&L, &tt, &st, &o);
        trav = &tt;
    } else {
        tree_build(&st, &S, o.maxs);
        tree_build(&tt, &T, o.maxt);
        lists_make(&L, &st, &tt, &o);
        trav = &st;
    }
    *units = L.units;
    *nodes = trav->n;
    long cnt = 0;
    for (int u = 0; u < L.units; u++) {
        ivec *kinds[4] = {&L.pp[u], &L.ap[u], &L.pc[u], &L.cp[u]};
        for (int k = 0; k < 4; k++) {
            for (int e = 0; e < kinds[k]->n; e++) {
                if (cnt < cap) {
                    entries[3 * cnt] = u; entries[3 * cnt + 1] = k; entries[3 * cnt + 2] = kinds[k]->v[e];
                }
                cnt++;
            }
        }
    }
    lists_free(&L);
    ot_free(&st); ot_free(&tt);
    op_free(&S); op_free(&T);
    return cnt <= cap ? cnt : -1;
}
