/*
 * bt_lists.c -- MAC-driven interaction lists and their device work layout.
 *
 * The traversals restate pc_compute_interaction_list and
 * cc_compute_interaction_list (src/interaction_lists/interaction_lists.c:464-533,
 * 537-748) with the same comparisons in the same FP64 arithmetic, so list
 * membership and order equal the reference's.  The lists are then reshaped
 * for the GPU so that every output value has exactly one writer:
 *   - per target leaf: the source clusters (PC) and source nodes (PP) acting
 *     on its particles, with CC-mode lists of ancestor target nodes pushed
 *     down to the leaves;
 *   - per target node: the source clusters (M2L) and source nodes (CP) acting
 *     on its grid.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "bt_host.h"

typedef struct { int n, cap; int *v; } ivec;

static void iv_push(ivec *a, int x)
{
    if (a->n == a->cap) {
        a->cap = a->cap ? a->cap * 2 : 16;
        a->v = (int *)realloc(a->v, sizeof(int) * (size_t)a->cap);
    }
    a->v[a->n++] = x;
}

void bt_csr_free(bt_csr *c)
{
    free(c->off); free(c->idx);
    memset(c, 0, sizeof(*c));
}

static void csr_from_vecs(bt_csr *c, ivec *v, int rows)
{
    c->rows = rows;
    c->off = malloc(sizeof(int64_t) * (size_t)(rows + 1));
    c->off[0] = 0;
    for (int r = 0; r < rows; r++) c->off[r + 1] = c->off[r] + v[r].n;
    c->idx = malloc(sizeof(int) * (size_t)(c->off[rows] > 0 ? c->off[rows] : 1));
    for (int r = 0; r < rows; r++) {
        if (v[r].n) memcpy(c->idx + c->off[r], v[r].v, sizeof(int) * (size_t)v[r].n);
        free(v[r].v);
    }
    free(v);
}

/* pc_compute_interaction_list: depth-first, children in order; an explicit
 * stack visits nodes in the same order as the reference's recursion. */
static void pc_traverse(const bt_tree *t, int root, double br, double bx, double by, double bz,
                        const bt_params *o, ivec *ap, ivec *pp, int *stack)
{
    int sp = 0;
    if (root < 0) return;
    stack[sp++] = root;
    double thr = o->size_check * o->P;
    while (sp) {
        int node = stack[--sp];
        double tx = bx - t->xm[node], ty = by - t->ym[node], tz = bz - t->zm[node];
        double dist = sqrt(tx * tx + ty * ty + tz * tz);
        if (((t->rad[node] + br) < dist * o->theta) && (t->rad[node] != 0.00) && (thr < t->numpar[node])) {
            iv_push(ap, node);
        } else if (t->nchild[node] == 0) {
            iv_push(pp, node);
        } else {
            for (int i = t->nchild[node] - 1; i >= 0; i--) stack[sp++] = t->child[8 * node + i];
        }
    }
}

typedef struct { ivec *pp, *ap, *pc, *cp; } cc_out;

static void cc_traverse(const bt_tree *S, int s, const bt_tree *T, int t, const bt_params *o, cc_out *L)
{
    int size_check = (int)(o->size_check * o->P);
    double tx = T->xm[t] - S->xm[s], ty = T->ym[t] - S->ym[s], tz = T->zm[t] - S->zm[s];
    double dist = sqrt(tx * tx + ty * ty + tz * tz);
    if ((S->rad[s] + T->rad[t]) < dist * o->theta) {
        if (S->numpar[s] <= size_check && T->numpar[t] <= size_check) iv_push(&L->pp[t], s);
        else if (S->numpar[s] <= size_check) iv_push(&L->cp[t], s);
        else if (T->numpar[t] <= size_check) iv_push(&L->pc[t], s);
        else iv_push(&L->ap[t], s);
        return;
    }
    if (T->nchild[t] == 0 && S->nchild[s] == 0) {
        iv_push(&L->pp[t], s);
    } else if (S->nchild[s] == 0) {
        for (int i = 0; i < T->nchild[t]; i++) cc_traverse(S, s, T, T->child[8 * t + i], o, L);
    } else if (T->nchild[t] == 0) {
        for (int i = 0; i < S->nchild[s]; i++) cc_traverse(S, S->child[8 * s + i], T, t, o, L);
    } else if (S->numpar[s] < T->numpar[t]) {
        for (int i = 0; i < T->nchild[t]; i++) cc_traverse(S, s, T, T->child[8 * t + i], o, L);
    } else {
        for (int i = 0; i < S->nchild[s]; i++) cc_traverse(S, S->child[8 * s + i], T, t, o, L);
    }
}

static ivec *vecs(int n) { return calloc((size_t)(n > 0 ? n : 1), sizeof(ivec)); }

static void empty_csr(bt_csr *c, int rows)
{
    csr_from_vecs(c, vecs(rows), rows);
}

void bt_csr_empty(bt_csr *c, int rows)
{
    empty_csr(c, rows);
}

/* Invert a CSR (rows = units, idx = columns in [0, ncols)) to rows = columns,
 * keeping row order, and optionally mapping each column through colmap. */
static void csr_invert(const bt_csr *a, int ncols, const int *colmap, int nrows_out, bt_csr *out)
{
    ivec *v = vecs(nrows_out);
    for (int r = 0; r < a->rows; r++)
        for (int64_t k = a->off[r]; k < a->off[r + 1]; k++) {
            int c = a->idx[k];
            int row = colmap ? colmap[c] : c;
            (void)ncols;
            iv_push(&v[row], r);
        }
    csr_from_vecs(out, v, nrows_out);
}

void bt_plan_lists(bt_plan *pl)
{
    const bt_params *o = &pl->prm;
    if (o->ctype == 1 || o->ctype == 2) {
        /* PC: traverse the source tree for every target batch; CP: traverse
         * the target tree for every source batch (treedriver.c:181, :463). */
        const bt_tree *trav = (o->ctype == 1) ? &pl->st : &pl->tt;
        const bt_tree *bat = (o->ctype == 1) ? &pl->tt : &pl->st;
        int nb = bat->nleaves;
        ivec *ap = vecs(nb), *pp = vecs(nb);
#pragma omp parallel
        {
            int *stack = malloc(sizeof(int) * (size_t)(8 * trav->n + 8));
#pragma omp for schedule(dynamic, 8)
            for (int i = 0; i < nb; i++) {
                /* the batch's system: the other side's tree of the same system */
                int lo = 0, hi = bat->nroots;
                while (hi - lo > 1) {
                    int m = (lo + hi) / 2;
                    if (bat->leaf_off[m] <= i) lo = m; else hi = m;
                }
                int b = bat->leaves[i];
                pc_traverse(trav, trav->roots[lo], bat->rad[b], bat->xm[b], bat->ym[b], bat->zm[b], o, &ap[i],
                            &pp[i], stack);
            }
            free(stack);
        }
        csr_from_vecs(&pl->ap, ap, nb);
        csr_from_vecs(&pl->pp, pp, nb);
        empty_csr(&pl->pc, nb);
        empty_csr(&pl->cp, nb);
    } else {
        int nt = pl->tt.n;
        cc_out L = {vecs(nt), vecs(nt), vecs(nt), vecs(nt)};
        /* one dual traversal per system (src/interaction_lists/interaction_lists.c:537-748) */
#pragma omp parallel for schedule(dynamic, 1)
        for (int k = 0; k < pl->st.nroots; k++)
            if (pl->st.roots[k] >= 0 && pl->tt.roots[k] >= 0)
                cc_traverse(&pl->st, pl->st.roots[k], &pl->tt, pl->tt.roots[k], o, &L);
        csr_from_vecs(&pl->pp, L.pp, nt);
        csr_from_vecs(&pl->ap, L.ap, nt);
        csr_from_vecs(&pl->pc, L.pc, nt);
        csr_from_vecs(&pl->cp, L.cp, nt);
    }

    bt_plan_work_lists(pl);
}

/* Device-shaped work lists from the reference-shaped lists (pl->ap, pp, pc,
 * cp), whichever traversal made them. */
void bt_plan_work_lists(bt_plan *pl)
{
    const bt_params *o = &pl->prm;
    const bt_tree *T = &pl->tt;
    pl->n_units_t = T->nleaves;
    int *leaf_of = malloc(sizeof(int) * (size_t)(T->n > 0 ? T->n : 1));
    for (int i = 0; i < T->n; i++) leaf_of[i] = -1;
    for (int i = 0; i < T->nleaves; i++) leaf_of[T->leaves[i]] = i;

    if (o->ctype == 1) {
        /* batches are the target leaves in the same order */
        bt_csr *srcs[2] = {&pl->ap, &pl->pp};
        bt_csr *dsts[2] = {&pl->t_approx, &pl->t_direct};
        for (int k = 0; k < 2; k++) {
            bt_csr *d = dsts[k];
            d->rows = srcs[k]->rows;
            d->off = malloc(sizeof(int64_t) * (size_t)(d->rows + 1));
            memcpy(d->off, srcs[k]->off, sizeof(int64_t) * (size_t)(d->rows + 1));
            int64_t m = d->off[d->rows];
            d->idx = malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
            if (m) memcpy(d->idx, srcs[k]->idx, sizeof(int) * (size_t)m);
        }
        empty_csr(&pl->g_cc, T->n);
        empty_csr(&pl->g_cp, T->n);
    } else if (o->ctype == 2) {
        /* units are source batches; entries are target nodes (CP) and target
         * leaves (PP); invert so each target node/leaf owns its sources, given
         * as source-tree node indices (the batches are the source leaves). */
        bt_csr tmp_cp, tmp_pp;
        csr_invert(&pl->ap, T->n, NULL, T->n, &tmp_cp);
        csr_invert(&pl->pp, T->n, leaf_of, T->nleaves, &tmp_pp);
        for (int64_t k = 0; k < tmp_cp.off[tmp_cp.rows]; k++) tmp_cp.idx[k] = pl->st.leaves[tmp_cp.idx[k]];
        for (int64_t k = 0; k < tmp_pp.off[tmp_pp.rows]; k++) tmp_pp.idx[k] = pl->st.leaves[tmp_pp.idx[k]];
        pl->g_cp = tmp_cp;
        pl->t_direct = tmp_pp;
        empty_csr(&pl->t_approx, T->nleaves);
        empty_csr(&pl->g_cc, T->n);
    } else {
        /* CC: grid-side lists per target node as built; particle-side lists
         * of every ancestor pushed down to each target leaf. */
        bt_csr *srcs[2] = {&pl->ap, &pl->cp};
        bt_csr *dsts[2] = {&pl->g_cc, &pl->g_cp};
        for (int k = 0; k < 2; k++) {
            bt_csr *d = dsts[k];
            d->rows = srcs[k]->rows;
            d->off = malloc(sizeof(int64_t) * (size_t)(d->rows + 1));
            memcpy(d->off, srcs[k]->off, sizeof(int64_t) * (size_t)(d->rows + 1));
            int64_t m = d->off[d->rows];
            d->idx = malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
            if (m) memcpy(d->idx, srcs[k]->idx, sizeof(int) * (size_t)m);
        }
        ivec *va = vecs(T->nleaves), *vd = vecs(T->nleaves);
        for (int u = 0; u < T->nleaves; u++) {
            for (int a = T->leaves[u]; a >= 0; a = T->parent[a]) {
                for (int64_t k = pl->pc.off[a]; k < pl->pc.off[a + 1]; k++) iv_push(&va[u], pl->pc.idx[k]);
                for (int64_t k = pl->pp.off[a]; k < pl->pp.off[a + 1]; k++) iv_push(&vd[u], pl->pp.idx[k]);
            }
        }
        csr_from_vecs(&pl->t_approx, va, T->nleaves);
        csr_from_vecs(&pl->t_direct, vd, T->nleaves);
    }
    free(leaf_of);
}

void bt_plan_free(bt_plan *pl)
{
    bt_parts_free(&pl->src);
    bt_parts_free(&pl->tgt);
    bt_tree_free(&pl->st);
    bt_tree_free(&pl->tt);
    bt_csr *c[8] = {&pl->pp, &pl->ap, &pl->pc, &pl->cp, &pl->t_approx, &pl->t_direct, &pl->g_cc, &pl->g_cp};
    for (int i = 0; i < 8; i++) bt_csr_free(c[i]);
    free(pl->a_deg);
    pl->a_deg = NULL;
}
