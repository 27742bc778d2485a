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
    memset(t, 0, sizeof(*t));
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

static int build_node(bt_tree *t, build_ctx *c, int b, int np, int level, int parent)
{
    bt_parts *p = c->p;
    tree_grow(t);
    int idx = t->n++;
    t->ibeg[idx] = b; t->numpar[idx] = np; t->level[idx] = level; t->parent[idx] = parent;
    t->nchild[idx] = 0;
    if (level + 1 > t->max_depth) t->max_depth = level + 1;

    /* bounding box of the node's particles (tree_linked_list.c:188-206) */
    const double *xs = p->x + b, *ys = p->y + b, *zs = p->z + b;
    double x0 = xs[0], x1 = xs[0], y0 = ys[0], y1 = ys[0], z0 = zs[0], z1 = zs[0];
    for (int i = 1; i < np; i++) {
        if (x0 > xs[i]) x0 = xs[i];
        if (x1 < xs[i]) x1 = xs[i];
        if (y0 > ys[i]) y0 = ys[i];
        if (y1 < ys[i]) y1 = ys[i];
        if (z0 > zs[i]) z0 = zs[i];
        if (z1 < zs[i]) z1 = zs[i];
    }
    double xl = x1 - x0, yl = y1 - y0, zl = z1 - z0;
    t->x0[idx] = x0; t->x1[idx] = x1; t->y0[idx] = y0; t->y1[idx] = y1; t->z0[idx] = z0; t->z1[idx] = z1;
    double xm = (x1 + x0) / 2.0, ym = (y1 + y0) / 2.0, zm = (z1 + z0) / 2.0;
    t->xm[idx] = xm; t->ym[idx] = ym; t->zm[idx] = zm;
    t->rad[idx] = sqrt(xl * xl + yl * yl + zl * zl) / 2.0;

    if (np <= c->maxpar) return idx;

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
    memset(code, 0, (size_t)np);
    int cnt[8] = {np, 0, 0, 0, 0, 0, 0, 0};
    int bit = 0;
    const double *ax[3] = {xs, ys, zs};
    double mid[3] = {xm, ym, zm};
    for (int a = 0; a < 3; a++) {
        if (!div[a]) continue;
        const double *v = ax[a];
        double m = mid[a];
        int newcnt[8] = {0};
        for (int i = 0; i < np; i++) {
            int part = code[i];
            int upper = (cnt[part] >= 2) ? !(v[i] <= m) : !(v[i] < m);
            code[i] = (unsigned char)(part | (upper << bit));
            newcnt[code[i]]++;
        }
        memcpy(cnt, newcnt, sizeof cnt);
        bit++;
    }
    int nslots = 1 << bit;
    /* Memory layout of the slots: each binary split keeps its lower part
     * first, so the first divided axis is the most significant position key
     * (the slot index with its bits reversed), while children are numbered
     * in slot order.  Same ranges as the reference's ibeg/iend. */
    int start[8], pos[8];
    {
        int off = 0;
        for (int key = 0; key < nslots; key++) {
            int s = 0;
            for (int k = 0; k < bit; k++) s |= ((key >> (bit - 1 - k)) & 1) << k;
            start[s] = off;
            off += cnt[s];
        }
    }
    memcpy(pos, start, sizeof pos);
    double *tx = c->tx + b, *ty = c->ty + b, *tz = c->tz + b, *tq = c->tq + b;
    int *to = c->to + b;
    double *px = p->x + b, *py = p->y + b, *pz = p->z + b, *pq = p->q + b;
    int *po = p->order + b;
    for (int i = 0; i < np; i++) {
        int d = pos[code[i]]++;
        tx[d] = px[i]; ty[d] = py[i]; tz[d] = pz[i]; tq[d] = pq[i]; to[d] = po[i];
    }
    memcpy(px, tx, sizeof(double) * (size_t)np);
    memcpy(py, ty, sizeof(double) * (size_t)np);
    memcpy(pz, tz, sizeof(double) * (size_t)np);
    memcpy(pq, tq, sizeof(double) * (size_t)np);
    memcpy(po, to, sizeof(int) * (size_t)np);

    /* A split that leaves every particle in one slot (all particles of an
     * over-full node at one point) would repeat forever; the reference
     * recurses without end there.  Keep such a node as a leaf. */
    for (int s = 0; s < nslots; s++)
        if (cnt[s] == np) return idx;

    int kids[8], nk = 0;
    for (int s = 0; s < nslots; s++) {
        if (cnt[s] == 0) continue;             /* empty children are skipped (tree_linked_list.c:266) */
        kids[nk++] = build_node(t, c, b + start[s], cnt[s], level + 1, idx);
    }
    t->nchild[idx] = nk;
    for (int i = 0; i < nk; i++) t->child[8 * idx + i] = kids[i];
    return idx;
}

static void collect(bt_tree *t, int idx, int *nleaf, int *lvl_fill)
{
    if (t->nchild[idx] == 0) { t->leaves[(*nleaf)++] = idx; return; }
    int l = t->level[idx];
    t->lvl_nodes[t->lvl_off[l] + lvl_fill[l]++] = idx;
    for (int i = 0; i < t->nchild[idx]; i++) collect(t, t->child[8 * idx + i], nleaf, lvl_fill);
}

void bt_tree_build(bt_tree *t, bt_parts *p, int maxparnode)
{
    memset(t, 0, sizeof(*t));
    t->max_depth = 1;
    if (p->n <= 0) return;
    build_ctx c;
    size_t m = (size_t)p->n;
    c.p = p;
    c.tx = malloc(sizeof(double) * m); c.ty = malloc(sizeof(double) * m);
    c.tz = malloc(sizeof(double) * m); c.tq = malloc(sizeof(double) * m);
    c.to = malloc(sizeof(int) * m);
    c.code = malloc(m);
    c.maxpar = maxparnode;
    build_node(t, &c, 0, p->n, 0, -1);
    free(c.tx); free(c.ty); free(c.tz); free(c.tq); free(c.to); free(c.code);

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
    collect(t, 0, &nl, lvl_cnt);
    free(lvl_cnt);
}

void bt_cheb_nodes(int n, double a0, double a1, double *out)
{
    for (int i = 0; i <= n; i++) {
        double tt = cos(i * M_PI / n);
        out[i] = a0 + (tt + 1.0) / 2.0 * (a1 - a0);
    }
}
