/*
 * ref_sampled.c -- the reference's particle-cluster treecode with its setup
 * and its per-batch evaluation as separate calls.
 *
 * TEST INFRASTRUCTURE (the parity checker and the CPU baseline), compiled by
 * `make ref` together with the reference BaryTree sources into
 * oracle/_ref/libBaryTree_refsample.so.  It calls the reference's own
 * routines in the order of treedriver's particle-cluster branch
 * (src/drivers/treedriver.c:346-460, one rank):
 *
 *   RunParams_Setup, Particles_Validate, Particles_ConstructOrder,
 *   Tree_Sources_Construct, Batches_Targets_Construct,
 *   Clusters_Sources_Construct, InteractionLists_Make
 *
 * once (refs_setup), and then InteractionCompute_PC
 * (src/interaction_compute/interaction_compute_pc.c:29-649) on any chosen
 * subset of the target batches (refs_eval).  A batch's potentials depend only
 * on the batch, its two lists and the source tree's proxies, so every batch
 * evaluated here holds exactly the values a full BaryTreeInterface call gives
 * it.  That makes two things possible at sizes where a full CPU call takes
 * tens of minutes: parity of sampled batches against the reference itself,
 * and the reference's whole-system time as setup + evaluation, the
 * evaluation measured on a strided sample of the batches.
 *
 * refs_eval hands the chosen batches to OpenMP threads, one batch per call of
 * InteractionCompute_PC: batches write disjoint targets, and the reference's
 * compute routines keep no state between calls, so this is the reference's
 * evaluation split over host cores (the reference itself is serial).
 */
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <omp.h>

#include "particles/struct_particles.h"
#include "particles/particles.h"
#include "run_params/struct_run_params.h"
#include "run_params/run_params.h"
#include "tree/struct_tree.h"
#include "tree/tree.h"
#include "tree/batches.h"
#include "clusters/struct_clusters.h"
#include "clusters/clusters.h"
#include "interaction_lists/struct_interaction_lists.h"
#include "interaction_lists/interaction_lists.h"
#include "interaction_compute/interaction_compute.h"

typedef struct {
    struct Particles S, T;
    struct RunParams *rp;
    struct Tree *tree, *batches;
    struct Clusters *clusters;
    struct InteractionLists *lists;
    double *pot;                 /* target tree order */
} refs_handle;

static double wall(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static double *dup(const double *a, int n)
{
    double *b = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    if (n > 0) memcpy(b, a, sizeof(double) * (size_t)n);
    return b;
}

/* Setup of one particle-cluster system (skipping).  phase_seconds receives
 * the reference's own setup phases: [0] source tree, [1] target batches,
 * [2] source proxies (upward pass), [3] interaction lists.  The inputs are
 * copied (the reference permutes its arrays in place). */
void *refs_setup(int nt, int ns, const double *tx, const double *ty, const double *tz,
                 const double *sx, const double *sy, const double *sz, const double *sq,
                 int kernel, int nkp, const double *kp, int approximation, double theta, int degree,
                 int maxs, int maxt, double size_check, double *phase_seconds)
{
    refs_handle *h = calloc(1, sizeof(refs_handle));
    RunParams_Setup(&h->rp, (KERNEL)kernel, nkp, (double *)kp, (APPROXIMATION)approximation, SKIPPING,
                    PARTICLE_CLUSTER, theta, degree, maxs, maxt, size_check, -1.0, 0);
    h->S.num = ns;
    h->S.x = dup(sx, ns); h->S.y = dup(sy, ns); h->S.z = dup(sz, ns); h->S.q = dup(sq, ns);
    h->T.num = nt;
    h->T.x = dup(tx, nt); h->T.y = dup(ty, nt); h->T.z = dup(tz, nt);
    RunParams_Validate(h->rp);
    Particles_Validate(&h->S, &h->T, h->rp);
    Particles_ConstructOrder(&h->S);
    Particles_ConstructOrder(&h->T);
    double t0 = wall();
    Tree_Sources_Construct(&h->tree, &h->S, h->rp);
    double t1 = wall();
    Batches_Targets_Construct(&h->batches, &h->T, h->rp);
    double t2 = wall();
    Clusters_Sources_Construct(&h->clusters, &h->S, h->tree, h->rp);
    double t3 = wall();
    InteractionLists_Make(&h->lists, h->tree, h->batches, h->rp);
    double t4 = wall();
    if (phase_seconds) {
        phase_seconds[0] = t1 - t0; phase_seconds[1] = t2 - t1;
        phase_seconds[2] = t3 - t2; phase_seconds[3] = t4 - t3;
    }
    h->pot = calloc((size_t)(nt > 0 ? nt : 1), sizeof(double));
    return h;
}

int refs_num_batches(void *vh)
{
    return ((refs_handle *)vh)->batches->numnodes;
}

/* Pointwise interactions of batch b, counted as the reference counts them
 * (src/drivers/treedriver.c:467-483): PP m*n_s, PC m*P. */
long long refs_batch_work(void *vh, int b)
{
    refs_handle *h = vh;
    long long m = h->batches->numpar[b], w = 0;
    for (int j = 0; j < h->lists->num_pp[b]; j++) w += m * h->tree->numpar[h->lists->pp_interactions[b][j]];
    w += m * (long long)h->lists->num_pc[b] * h->rp->interp_pts_per_cluster;
    return w;
}

int refs_batch_size(void *vh, int b)
{
    return ((refs_handle *)vh)->batches->numpar[b];
}

/* InteractionCompute_PC on the batches sel[0..nsel) with `threads` OpenMP
 * threads.  The potentials of those batches' targets are written into
 * out_caller (indexed in the caller's target order; other entries are left
 * alone); batch_seconds (may be NULL) receives each batch's own time on its
 * thread.  Returns the wall seconds of the evaluation. */
double refs_eval(void *vh, int nsel, const int *sel, int threads, double *out_caller, double *batch_seconds)
{
    refs_handle *h = vh;
    struct Tree *B = h->batches;
    struct InteractionLists *L = h->lists;
    double t0 = wall();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1)
    for (int k = 0; k < nsel; k++) {
        int b = sel[k];
        struct Tree one;
        memset(&one, 0, sizeof one);
        one.numnodes = 1;
        one.ibeg = &B->ibeg[b];
        one.iend = &B->iend[b];
        one.numpar = &B->numpar[b];
        struct InteractionLists l1;
        memset(&l1, 0, sizeof l1);
        l1.num_pc = &L->num_pc[b];
        l1.num_pp = &L->num_pp[b];
        l1.pc_interactions = &L->pc_interactions[b];
        l1.pp_interactions = &L->pp_interactions[b];
        double tb = wall();
        for (int i = B->ibeg[b] - 1; i < B->iend[b]; i++) h->pot[i] = 0.0;
        InteractionCompute_PC(h->pot, h->tree, &one, &l1, &h->S, &h->T, h->clusters, h->rp);
        if (batch_seconds) batch_seconds[k] = wall() - tb;
    }
    double t1 = wall();
    if (out_caller)
        for (int k = 0; k < nsel; k++) {
            int b = sel[k];
            for (int i = B->ibeg[b] - 1; i < B->iend[b]; i++) out_caller[h->T.order[i] - 1] = h->pot[i];
        }
    return t1 - t0;
}

void refs_free(void *vh)
{
    refs_handle *h = vh;
    if (!h) return;
    InteractionLists_Free(&h->lists);
    Clusters_Free_Win(&h->clusters);     /* allocated as MPI window memory (clusters.c:76-87) */
    Batches_Free(&h->batches);
    Tree_Free(&h->tree);
    free(h->S.x); free(h->S.y); free(h->S.z); free(h->S.q);
    free(h->T.x); free(h->T.y); free(h->T.z);
    if (h->S.sources_w_dummy) free(h->S.w);
    if (h->T.targets_q_dummy) free(h->T.q);
    free(h->S.order); free(h->T.order);
    free(h->pot);
    RunParams_Free(&h->rp);
    free(h);
}
