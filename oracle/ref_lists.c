/*
 * ref_lists.c -- dump trees and interaction lists from the reference build.
 *
 * TEST INFRASTRUCTURE, compiled by `make ref` together with the reference
 * BaryTree sources into oracle/_ref/libBaryTree_reflists.so.  It calls the
 * reference's own internal routines (Tree_*_Construct, Batches_*_Construct,
 * InteractionLists_Make; src/tree/tree.h, src/tree/batches.h,
 * src/interaction_lists/interaction_lists.h:9) and flattens their output in
 * the same canonical form as bto_lists / bto_tree in bt_oracle.c.
 */
#include <stdlib.h>
#include <string.h>

#include "particles/struct_particles.h"
#include "particles/particles.h"
#include "run_params/struct_run_params.h"
#include "run_params/run_params.h"
#include "tree/struct_tree.h"
#include "tree/tree.h"
#include "tree/batches.h"
#include "interaction_lists/struct_interaction_lists.h"
#include "interaction_lists/interaction_lists.h"

static struct Particles *mkpart(int n, const double *x, const double *y, const double *z)
{
    struct Particles *p = calloc(1, sizeof(struct Particles));
    p->num = n;
    p->x = malloc(sizeof(double) * (n > 0 ? n : 1));
    p->y = malloc(sizeof(double) * (n > 0 ? n : 1));
    p->z = malloc(sizeof(double) * (n > 0 ? n : 1));
    p->q = calloc(n > 0 ? n : 1, sizeof(double));
    p->w = calloc(n > 0 ? n : 1, sizeof(double));
    memcpy(p->x, x, sizeof(double) * n);
    memcpy(p->y, y, sizeof(double) * n);
    memcpy(p->z, z, sizeof(double) * n);
    Particles_ConstructOrder(p);
    return p;
}

static void freepart(struct Particles *p)
{
    free(p->x); free(p->y); free(p->z); free(p->q); free(p->w); free(p->order); free(p);
}

int refl_tree(int n, const double *x, const double *y, const double *z, int maxparnode,
              int *ints, double *dbl, int cap)
{
    struct Particles *p = mkpart(n, x, y, z);
    struct RunParams *rp = NULL;
    RunParams_Setup(&rp, COULOMB, 0, NULL, LAGRANGE, SKIPPING, PARTICLE_CLUSTER,
                    0.5, 1, maxparnode, maxparnode, 1.0, -1.0, 0);
    struct Tree *t = NULL;
    Tree_Sources_Construct(&t, p, rp);
    int nn = t->numnodes;
    if (nn <= cap) {
        for (int i = 0; i < nn; i++) {
            ints[4 * i] = t->ibeg[i]; ints[4 * i + 1] = t->iend[i];
            ints[4 * i + 2] = t->num_children[i]; ints[4 * i + 3] = 0;
            double d[7] = {t->x_min[i], t->x_max[i], t->y_min[i], t->y_max[i], t->z_min[i], t->z_max[i], t->radius[i]};
            memcpy(dbl + 7 * i, d, sizeof d);
        }
    }
    Tree_Free(&t);
    RunParams_Free(&rp);
    freepart(p);
    return nn <= cap ? nn : -1;
}

/* The reference's particle permutation after its tree build: order[i] =
 * 0-based input index of sorted particle i (Particles_ConstructOrder,
 * src/particles/particles.c:138-144, permuted by the partition). */
int refl_tree_order(int n, const double *x, const double *y, const double *z, int maxparnode, int *order)
{
    struct Particles *p = mkpart(n, x, y, z);
    struct RunParams *rp = NULL;
    RunParams_Setup(&rp, COULOMB, 0, NULL, LAGRANGE, SKIPPING, PARTICLE_CLUSTER,
                    0.5, 1, maxparnode, maxparnode, 1.0, -1.0, 0);
    struct Tree *t = NULL;
    Tree_Sources_Construct(&t, p, rp);
    for (int i = 0; i < n; i++) order[i] = p->order[i] - 1;
    Tree_Free(&t);
    RunParams_Free(&rp);
    freepart(p);
    return 0;
}

long refl_lists(int numTargets, int numSources,
                const double *targetX, const double *targetY, const double *targetZ,
                const double *sourceX, const double *sourceY, const double *sourceZ,
                int compute_type, int approximation, double theta, int interpDegree,
                int maxPerSourceLeaf, int maxPerTargetLeaf, double sizeCheck,
                int *units, int *nodes, int *entries, long cap)
{
    struct Particles *S = mkpart(numSources, sourceX, sourceY, sourceZ);
    struct Particles *T = mkpart(numTargets, targetX, targetY, targetZ);
    struct RunParams *rp = NULL;
    RunParams_Setup(&rp, COULOMB, 0, NULL, (APPROXIMATION)approximation, SKIPPING, (COMPUTE_TYPE)compute_type,
                    theta, interpDegree, maxPerSourceLeaf, maxPerTargetLeaf, sizeCheck, -1.0, 0);
    struct Tree *tree = NULL, *other = NULL;
    struct InteractionLists *il = NULL;
    int nunits;
    if (compute_type == PARTICLE_CLUSTER) {
        Tree_Sources_Construct(&tree, S, rp);
        Batches_Targets_Construct(&other, T, rp);
        InteractionLists_Make(&il, tree, other, rp);
    } else if (compute_type == CLUSTER_PARTICLE) {
        Tree_Targets_Construct(&tree, T, rp);
        Batches_Sources_Construct(&other, S, rp);
        InteractionLists_Make(&il, tree, other, rp);
    } else {
        Tree_Sources_Construct(&tree, S, rp);
        Tree_Targets_Construct(&other, T, rp);
        InteractionLists_Make(&il, tree, other, rp);
    }
    nunits = other->numnodes;
    *units = nunits;
    *nodes = tree->numnodes;
    int *nap = compute_type == PARTICLE_CLUSTER ? il->num_pc : compute_type == CLUSTER_PARTICLE ? il->num_cp : il->num_cc;
    int **ap = compute_type == PARTICLE_CLUSTER ? il->pc_interactions
             : compute_type == CLUSTER_PARTICLE ? il->cp_interactions : il->cc_interactions;
    long cnt = 0;
    for (int u = 0; u < nunits; u++) {
        int *nk[4] = {il->num_pp, nap, NULL, NULL};
        int **lk[4] = {il->pp_interactions, ap, NULL, NULL};
        if (compute_type == CLUSTER_CLUSTER) {
            nk[2] = il->num_pc; lk[2] = il->pc_interactions;
            nk[3] = il->num_cp; lk[3] = il->cp_interactions;
        }
        for (int k = 0; k < 4; k++) {
            if (!nk[k]) continue;
            for (int e = 0; e < nk[k][u]; e++) {
                if (cnt < cap) {
                    entries[3 * cnt] = u; entries[3 * cnt + 1] = k; entries[3 * cnt + 2] = lk[k][u][e];
                }
                cnt++;
            }
        }
    }
    InteractionLists_Free(&il);    /* frees NULL kinds safely (src/utilities/array.h free_matrix) */
    if (compute_type == CLUSTER_CLUSTER) Tree_Free(&other);
    else Batches_Free(&other);
    Tree_Free(&tree);
    RunParams_Free(&rp);
    freepart(S); freepart(T);
    return cnt <= cap ? cnt : -1;
}
