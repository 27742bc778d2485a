/*
 * bt_tree.c -- run parameters, particle copies and the adaptive tree build.
 *
 * The tree reproduces the reference's node sets exactly
 * (TreeLinkedList_*_Construct, src/tree/tree_linked_list.c:16-280, with the
 * split rule of pc_partition_8/cp_partition_8, src/tree/partition.c:178-392),
 * because interaction-list membership depends only on each node's particle
 * set (its box, centre, radius and count).  The order of particles inside a
 * node is not observable in the lists, so instead of the reference's
 * repeated in-place binary Hoare partitions (src/tree/partition.c:14-175)
 * each node is split in one pass: every particle gets its child slot from
 * the same comparisons, then one stable counting scatter moves it.
 *
 * Nodes are numbered in pre-order and children kept in the reference's
 * ind[] order, so node indices equal the reference's.
 */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "bt_host.h"

/* RunParams_Setup (src/run_params/run_params.c:13-131): explicit parameters,
 * or theta/degree/size check/leaf sizes derived from beta in [0,1]. */
void bt_params_setup(bt_params *o, int kernel, int nkp, const double *kp, int sing, int approx,
                     int ctype, double theta, int degree, int maxs, int maxt, double sc, double beta,
                     int verbosity)
{
    memset(o, 0, sizeof(*o));
    o->kernel = kernel; o->sing = sing; o->approx = approx; o->ctype = ctype;
    o->kp = (nkp > 0 && kp) ? kp[0] : 0.0;
    o->kp2 = (nkp > 1 && kp) ? kp[1] : 0.0;
    o->nkp = kp ? nkp : 0;
    o->verbosity = verbosity;
    if (beta < 0 || beta > 1) {
        o->beta = -1;
        o->theta = theta; o->degree = degree; o->size_check = sc; o->maxs = maxs; o->maxt = maxt;
    } else {
        double tmin = 0.55, tmax = 0.95, es, nmin = 1, nmax, et = 3;
        o->beta = beta;
        if (ctype == 1 || ctype == 2) {
            es = 2;
            if (approx == 1) { o->size_check = 1.0; nmax = 12; }
            else { o->size_check = 4.0; nmax = 9; }
        } else {
            o->size_check = 1.0; es = 1.75; nmax = 12;
        }
        o->theta = tmax - (tmax - tmin) * pow(beta, es);
        o->degree = (int)(nmax - (nmax - nmin) * pow(1. - beta, et));
        /* CPU leaf sizes of the reference (run_params.c:107-119): the beta path
         * is defined by them, so keep them for identical trees and lists. */
        if (ctype == 1) { o->maxs = 50; o->maxt = 5; }
        else if (ctype == 2) { o->maxs = 5; o->maxt = 50; }
        else { o->maxs = 50; o->maxt = 50; }
    }
    o->P = (o->degree + 1) * (o->degree + 1) * (o->degree + 1);
}

void bt_parts_init(bt_parts *p, int n, const double *x, const double *y, const double *z, const double *q)
{
    size_t m = (size_t)(n > 0 ? n : 1);
    p->n = n;
    p->x = malloc(sizeof(double) * m);
    p->y = malloc(sizeof(double) * m);
    p->z = malloc(sizeof(double) * m);
    p->q = malloc(sizeof(double) * m);
    p->order = malloc(sizeof(int) * m);
    if (n > 0) {
        memcpy(p->x, x, sizeof(double) * (size_t)n);
        memcpy(p->y, y, sizeof(double) * (size_t)n);
        memcpy(p->z, z, sizeof(double) * (size_t)n);
        if (q) memcpy(p->q, q, sizeof(double) * (size_t)n);
        else memset(p->q, 0, sizeof(double) * (size_t)n);
    }
    for (int i = 0; i < n; i++) p->order[i] = i;
}

void bt_parts_free(bt_parts *p)
{
    free(p->x); free(p->y); free(p->z); free(p->q); free(p->order);
    memset(p, 0, sizeof(*p));
}

static void tree_grow(bt_tree *t)
{
    if (t->n < t->cap) return;
    int c = t->cap ? t->cap * 2 : 256;
#define G(f, T) t->f = (T *)realloc(t->f, sizeof(T) * (size_t)c)
    G(ibeg, int); G(numpar, int); G(nchild, int); G(parent, int); G(level, int);
    G(x0, double); G(x1, double); G(y0, double); G(y1, double); G(z0, double); G(z1, double);
    G(xm, double); G(ym, double); G(zm, double); G(rad, double);
#undef G
    t->child = (int *)realloc(t->child, sizeof(int) * 8 * (size_t)c);
    t->cap = c;
}

void bt_tree_free(bt_tree *t)
{
    free(t->ibeg); free(t->numpar); free(t->nchild); free(t->parent); free(t->level); free(t->child);
    free(t->x0); free(t->x1); free(t->y0); free(t->y1); free(t->z0); free(t->z1);
    free(t->xm); free(t->ym); free(t->zm); free(t->rad);
    free(t->leaves); free(t->lvl_off); free(t->lvl_nodes);
    free(t->roots); free(t->leaf_off);
    memset(t, 0, sizeof(*t));
}

void bt_tree_set_roots(bt_tree *t, int nsys)
{
    free(t->roots);
    t->nroots = nsys;
    t->roots = malloc(sizeof(int) * (size_t)(nsys > 0 ? nsys : 1));
    for (int k = 0; k < nsys; k++) t->roots[k] = -1;
}

typedef struct {
    bt_parts *p;
    double *tx, *ty, *tz, *tq;
    int *to;
    unsigned char *code;
    int maxpar;
} build_ctx;

/* Split rule of pc_partition_8 (src/tree/partition.c:178-227): which axes to
 * divide given the node extents and the child budget. */
static void divide_axes(double xl, double yl, double zl, int max_nc, int div[3])
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

/* One node of the level-synchronous build.  Nodes are created level by
 * level (breadth first) and renumbered to the reference's pre-order at the
 * end, so the build can split every node of a level concurrently. */
typedef struct {
    int ibeg, np, level, parent, nchild, child[8];
    int kid_b[8], kid_n[8];
    double box[6];                  /* x0, x1, y0, y1, z0, z1 */
} bnode;

/* Nodes at least this large are split with parallel loops; smaller nodes of
 * a level are split concurrently, one thread per node. */
#define BT_PAR_NODE 65536

static void split_node(bnode *nd, build_ctx *c, int par)
{
    bt_parts *p = c->p;
    const int b = nd->ibeg, np = nd->np;
    const double *xs = p->x + b, *ys = p->y + b, *zs = p->z + b;
    nd->nchild = 0;

    /* bounding box of the node's particles (tree_linked_list.c:188-206) */
    double x0 = xs[0], x1 = xs[0], y0 = ys[0], y1 = ys[0], z0 = zs[0], z1 = zs[0];
#pragma omp parallel for if (par) reduction(min : x0, y0, z0) reduction(max : x1, y1, z1)
    for (int i = 0; i < np; i++) {
        if (x0 > xs[i]) x0 = xs[i];
        if (x1 < xs[i]) x1 = xs[i];
        if (y0 > ys[i]) y0 = ys[i];
        if (y1 < ys[i]) y1 = ys[i];
        if (z0 > zs[i]) z0 = zs[i];
        if (z1 < zs[i]) z1 = zs[i];
    }
    nd->box[0] = x0; nd->box[1] = x1; nd->box[2] = y0; nd->box[3] = y1; nd->box[4] = z0; nd->box[5] = z1;
    if (np <= c->maxpar) return;

    double xl = x1 - x0, yl = y1 - y0, zl = z1 - z0;
    double mid[3] = {(x1 + x0) / 2.0, (y1 + y0) / 2.0, (z1 + z0) / 2.0};
    int max_nc = (np < 2 * c->maxpar) ? 2 : (np < 4 * c->maxpar) ? 4 : 8;
    int div[3];
    divide_axes(xl, yl, zl, max_nc, div);

    /* Child slot of every particle.  The reference splits the divided axes in
     * turn (x, y, z), each over the parts made by the previous splits; a part
     * of two or more particles sends {a <= mid} to the lower side, a part of
     * exactly one sends it lower only if a < mid (src/tree/partition.c:75-79).
     * The k-th divided axis sets bit k of the slot, which is the reference's
     * ind[] position (partition.c:229-282). */
    unsigned char *code = c->code + b;
#pragma omp parallel for if (par)
    for (int i = 0; i < np; i++) code[i] = 0;
    int cnt[8] = {np, 0, 0, 0, 0, 0, 0, 0};
    int bit = 0;
    const double *ax[3] = {xs, ys, zs};
    for (int a = 0; a < 3; a++) {
        if (!div[a]) continue;
        const double *v = ax[a];
        const double m = mid[a];
        int nc0 = cnt[0], nc1 = cnt[1], nc2 = cnt[2], nc3 = cnt[3];
        int pc[4] = {nc0, nc1, nc2, nc3};
        int newcnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma omp parallel for if (par) reduction(+ : newcnt[:8])
        for (int i = 0; i < np; i++) {
            int part = code[i];
            int upper = (pc[part] >= 2) ? !(v[i] <= m) : !(v[i] < m);
            int cd = part | (upper << bit);
            code[i] = (unsigned char)cd;
            newcnt[cd]++;
        }
        memcpy(cnt, newcnt, sizeof cnt);
        bit++;
    }
    int nslots = 1 << bit;

    /* A split that leaves every particle in one slot (all particles of an
     * over-full node at one point) would repeat forever; the reference
     * recurses without end there.  Keep such a node as a leaf. */
    for (int s = 0; s < nslots; s++)
        if (cnt[s] == np) return;

    /* Memory layout of the slots: each binary split keeps its lower part
     * first, so the first divided axis is the most significant position key
     * (the slot index with its bits reversed), while children are numbered
     * in slot order.  Same ranges as the reference's ibeg/iend. */
    int start[8];
    {
        int off = 0;
        for (int key = 0; key < nslots; key++) {
            int s = 0;
            for (int k = 0; k < bit; k++) s |= ((key >> (bit - 1 - k)) & 1) << k;
            start[s] = off;
            off += cnt[s];
        }
    }
    double *tx = c->tx + b, *ty = c->ty + b, *tz = c->tz + b, *tq = c->tq + b;
    int *to = c->to + b;
    double *px = p->x + b, *py = p->y + b, *pz = p->z + b, *pq = p->q + b;
    int *po = p->order + b;
    if (!par) {
        int pos[8];
        memcpy(pos, start, sizeof pos);
        for (int i = 0; i < np; i++) {
            int d = pos[code[i]]++;
            tx[d] = px[i]; ty[d] = py[i]; tz[d] = pz[i]; tq[d] = pq[i]; to[d] = po[i];
        }
    } else {
        /* stable parallel counting scatter: every thread scatters its
         * contiguous chunk behind the chunks of the threads before it */
        int nth = omp_get_max_threads();
        int (*tcnt)[8] = calloc((size_t)nth, sizeof(int[8]));
#pragma omp parallel num_threads(nth)
        {
            int t = omp_get_thread_num(), T = omp_get_num_threads();
            long lo = (long)np * t / T, hi = (long)np * (t + 1) / T;
            for (long i = lo; i < hi; i++) tcnt[t][code[i]]++;
#pragma omp barrier
#pragma omp single
            {
                for (int s = 0; s < 8; s++) {
                    int run = start[s];
                    for (int u = 0; u < T; u++) { int k = tcnt[u][s]; tcnt[u][s] = run; run += k; }
                }
            }
            int pos[8];
            memcpy(pos, tcnt[t], sizeof pos);
            for (long i = lo; i < hi; i++) {
                int d = pos[code[i]]++;
                tx[d] = px[i]; ty[d] = py[i]; tz[d] = pz[i]; tq[d] = pq[i]; to[d] = po[i];
            }
        }
        free(tcnt);
    }
#pragma omp parallel for if (par)
    for (int i = 0; i < np; i++) {
        px[i] = tx[i]; py[i] = ty[i]; pz[i] = tz[i]; pq[i] = tq[i]; po[i] = to[i];
    }
    for (int s = 0; s < nslots; s++) {
        if (cnt[s] == 0) continue;             /* empty children are skipped (tree_linked_list.c:266) */
        nd->kid_b[nd->nchild] = b + start[s];
        nd->kid_n[nd->nchild] = cnt[s];
        nd->nchild++;
    }
}

static void collect(bt_tree *t, int idx, int *nleaf, int *lvl_fill)
{
    if (t->nchild[idx] == 0) { t->leaves[(*nleaf)++] = idx; return; }
    int l = t->level[idx];
    t->lvl_nodes[t->lvl_off[l] + lvl_fill[l]++] = idx;
    for (int i = 0; i < t->nchild[idx]; i++) collect(t, t->child[8 * idx + i], nleaf, lvl_fill);
}

static int preorder(const bnode *nodes, int i, int next, int *pre)
{
    pre[i] = next++;
    for (int k = 0; k < nodes[i].nchild; k++) next = preorder(nodes, nodes[i].child[k], next, pre);
    return next;
}

void bt_tree_alloc(bt_tree *t, int n)
{
    t->cap = 0;
    t->n = 0;
    while (t->cap < n) {
        t->n = t->cap;          /* tree_grow grows when the arrays are full */
        tree_grow(t);
    }
    t->n = n;
}

void bt_tree_finish(bt_tree *t)
{
    /* leaves and per-level non-leaf lists, DFS order (src/tree/tree.c:122-153) */
    int nleaf = 0;
    int *lvl_cnt = calloc((size_t)t->max_depth + 1, sizeof(int));
    for (int i = 0; i < t->n; i++) {
        if (t->nchild[i] == 0) nleaf++;
        else lvl_cnt[t->level[i]]++;
    }
    t->nleaves = nleaf;
    t->leaves = malloc(sizeof(int) * (size_t)(nleaf > 0 ? nleaf : 1));
    t->lvl_off = malloc(sizeof(int) * (size_t)(t->max_depth + 1));
    t->lvl_off[0] = 0;
    for (int l = 0; l < t->max_depth; l++) t->lvl_off[l + 1] = t->lvl_off[l] + lvl_cnt[l];
    t->lvl_nodes = malloc(sizeof(int) * (size_t)(t->lvl_off[t->max_depth] + 1));
    memset(lvl_cnt, 0, sizeof(int) * (size_t)(t->max_depth + 1));
    int nl = 0;
    t->leaf_off = malloc(sizeof(int) * (size_t)(t->nroots + 1));
    for (int k = 0; k < t->nroots; k++) {
        t->leaf_off[k] = nl;
        if (t->roots[k] >= 0) collect(t, t->roots[k], &nl, lvl_cnt);
    }
    t->leaf_off[t->nroots] = nl;
    free(lvl_cnt);
}

void bt_tree_build(bt_tree *t, bt_parts *p, int maxparnode)
{
    int64_t off[2] = {0, p->n};
    bt_forest_build(t, p, 1, off, maxparnode);
}

void bt_forest_build(bt_tree *t, bt_parts *p, int nsys, const int64_t *sys_off, int maxparnode)
{
    memset(t, 0, sizeof(*t));
    t->max_depth = 1;
    bt_tree_set_roots(t, nsys);
    if (p->n <= 0) {
        t->leaf_off = calloc((size_t)nsys + 1, sizeof(int));
        return;
    }
    build_ctx c;
    size_t m = (size_t)p->n;
    c.p = p;
    c.tx = malloc(sizeof(double) * m); c.ty = malloc(sizeof(double) * m);
    c.tz = malloc(sizeof(double) * m); c.tq = malloc(sizeof(double) * m);
    c.to = malloc(sizeof(int) * m);
    c.code = malloc(m);
    c.maxpar = maxparnode;

    int cap = 1024 + nsys, n = 0;
    bnode *nodes = malloc(sizeof(bnode) * (size_t)cap);
    int *root_node = malloc(sizeof(int) * (size_t)nsys);
    for (int k = 0; k < nsys; k++) {
        root_node[k] = -1;
        if (sys_off[k + 1] <= sys_off[k]) continue;
        memset(&nodes[n], 0, sizeof(bnode));
        nodes[n].ibeg = (int)sys_off[k]; nodes[n].np = (int)(sys_off[k + 1] - sys_off[k]);
        nodes[n].level = 0; nodes[n].parent = -1;
        root_node[k] = n++;
    }
    int lo = 0, hi = n, depth = 1;
    while (lo < hi) {
        for (int i = lo; i < hi; i++)
            if (nodes[i].np >= BT_PAR_NODE) split_node(&nodes[i], &c, 1);
#pragma omp parallel for schedule(dynamic, 2)
        for (int i = lo; i < hi; i++)
            if (nodes[i].np < BT_PAR_NODE) split_node(&nodes[i], &c, 0);
        for (int i = lo; i < hi; i++) {
            for (int k = 0; k < nodes[i].nchild; k++) {
                if (n == cap) { cap *= 2; nodes = realloc(nodes, sizeof(bnode) * (size_t)cap); }
                bnode *ch = &nodes[n];
                memset(ch, 0, sizeof(bnode));
                ch->ibeg = nodes[i].kid_b[k]; ch->np = nodes[i].kid_n[k];
                ch->level = nodes[i].level + 1; ch->parent = i;
                nodes[i].child[k] = n;
                if (ch->level + 1 > depth) depth = ch->level + 1;
                n++;
            }
        }
        lo = hi; hi = n;
    }
    free(c.tx); free(c.ty); free(c.tz); free(c.tq); free(c.to); free(c.code);

    /* pre-order numbering (TreeLinkedList_SetIndex, src/tree/tree_linked_list.c:284-293),
     * system after system */
    int *pre = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    {
        int next = 0;
        for (int k = 0; k < nsys; k++)
            if (root_node[k] >= 0) {
                t->roots[k] = next;
                next = preorder(nodes, root_node[k], next, pre);
            }
    }
    free(root_node);
    bt_tree_alloc(t, n);
    t->max_depth = depth;
    for (int i = 0; i < n; i++) {
        const bnode *nd = &nodes[i];
        int k = pre[i];
        t->ibeg[k] = nd->ibeg; t->numpar[k] = nd->np; t->level[k] = nd->level;
        t->parent[k] = nd->parent >= 0 ? pre[nd->parent] : -1;
        t->nchild[k] = nd->nchild;
        for (int j = 0; j < nd->nchild; j++) t->child[8 * k + j] = pre[nd->child[j]];
        double x0 = nd->box[0], x1 = nd->box[1], y0 = nd->box[2], y1 = nd->box[3], z0 = nd->box[4], z1 = nd->box[5];
        double xl = x1 - x0, yl = y1 - y0, zl = z1 - z0;
        t->x0[k] = x0; t->x1[k] = x1; t->y0[k] = y0; t->y1[k] = y1; t->z0[k] = z0; t->z1[k] = z1;
        t->xm[k] = (x1 + x0) / 2.0; t->ym[k] = (y1 + y0) / 2.0; t->zm[k] = (z1 + z0) / 2.0;
        t->rad[k] = sqrt(xl * xl + yl * yl + zl * zl) / 2.0;
    }
    free(pre);
    free(nodes);

    bt_tree_finish(t);
}

void bt_tree_copy(bt_tree *dst, const bt_tree *src)
{
    memset(dst, 0, sizeof(*dst));
    dst->max_depth = 1;
    if (src->roots) {
        bt_tree_set_roots(dst, src->nroots);
        memcpy(dst->roots, src->roots, sizeof(int) * (size_t)src->nroots);
        dst->leaf_off = malloc(sizeof(int) * (size_t)(src->nroots + 1));
        memcpy(dst->leaf_off, src->leaf_off, sizeof(int) * (size_t)(src->nroots + 1));
    }
    if (src->n <= 0 || !src->lvl_off) return;
    int n = src->n;
    while (dst->cap < n) {
        dst->n = dst->cap;
        tree_grow(dst);
    }
    dst->n = n;
    dst->max_depth = src->max_depth;
    dst->nleaves = src->nleaves;
#define C(f) memcpy(dst->f, src->f, sizeof(*src->f) * (size_t)n)
    C(ibeg); C(numpar); C(nchild); C(parent); C(level);
    C(x0); C(x1); C(y0); C(y1); C(z0); C(z1); C(xm); C(ym); C(zm); C(rad);
#undef C
    memcpy(dst->child, src->child, sizeof(int) * 8 * (size_t)n);
    dst->leaves = malloc(sizeof(int) * (size_t)(src->nleaves > 0 ? src->nleaves : 1));
    memcpy(dst->leaves, src->leaves, sizeof(int) * (size_t)src->nleaves);
    dst->lvl_off = malloc(sizeof(int) * (size_t)(src->max_depth + 1));
    memcpy(dst->lvl_off, src->lvl_off, sizeof(int) * (size_t)(src->max_depth + 1));
    int nl = src->lvl_off[src->max_depth];
    dst->lvl_nodes = malloc(sizeof(int) * (size_t)(nl + 1));
    memcpy(dst->lvl_nodes, src->lvl_nodes, sizeof(int) * (size_t)nl);
}

void bt_cheb_nodes(int n, double a0, double a1, double *out)
{
    for (int i = 0; i <= n; i++) {
        double tt = cos(i * M_PI / n);
        out[i] = a0 + (tt + 1.0) / 2.0 * (a1 - a0);
    }
}
