/* bt_compat.c -- BaryTree's internal driver interface (RunParams_*,
 * treedriver, directdriver) on top of the library's own entry points, so
 * programs written against the reference's drivers link unchanged. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <time.h>

#include "../../include/barytree_compat.h"

static double wall_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* run_params.c:13-131.  The beta mapping matches bt_params_setup, which the
 * entry points use, so a struct built here describes the same run. */
void RunParams_Setup(struct RunParams **run_params_addr, KERNEL kernel, int num_kernel_params,
                     double *kernel_params, APPROXIMATION approximation, SINGULARITY singularity,
                     COMPUTE_TYPE compute_type, double theta, int interp_degree, int max_per_source_leaf,
                     int max_per_target_leaf, double size_check_factor, double beta, int verbosity)
{
    RunParams_Free(run_params_addr);
    struct RunParams *p = calloc(1, sizeof(struct RunParams));
    *run_params_addr = p;
    if (!p) return;
    p->verbosity = verbosity;
    p->kernel = kernel;
    p->num_kernel_params = num_kernel_params;
    if (num_kernel_params > 0) {
        p->kernel_params = malloc(sizeof(double) * (size_t)num_kernel_params);
        for (int i = 0; i < num_kernel_params; i++) p->kernel_params[i] = kernel_params[i];
    }
    p->approximation = approximation;
    p->singularity = singularity;
    p->compute_type = compute_type;
    if (beta < 0 || beta > 1) {
        p->beta = -1;
        p->theta = theta;
        p->interp_degree = interp_degree;
        p->size_check_factor = size_check_factor;
        p->max_per_source_leaf = max_per_source_leaf;
        p->max_per_target_leaf = max_per_target_leaf;
    } else {
        /* theta falls from 0.95 to 0.55 as beta^s, the degree rises from 1 to
         * n_max as 1 - (1-beta)^3; PC/CP use s = 2 (n_max 12 Lagrange, 9
         * Hermite, size check 1 and 4), CC uses s = 1.75 and n_max 12. */
        const int pc_cp = compute_type == PARTICLE_CLUSTER || compute_type == CLUSTER_PARTICLE;
        const double es = pc_cp ? 2.0 : 1.75;
        const double nmax = (pc_cp && approximation != LAGRANGE) ? 9.0 : 12.0;
        p->beta = beta;
        p->size_check_factor = (pc_cp && approximation != LAGRANGE) ? 4.0 : 1.0;
        const double tmin = 0.55, tmax = 0.95;   /* (tmax - tmin) rounds as in the reference */
        p->theta = tmax - (tmax - tmin) * pow(beta, es);
        p->interp_degree = (int)(nmax - (nmax - 1.0) * pow(1. - beta, 3.0));
        if (compute_type == PARTICLE_CLUSTER) { p->max_per_source_leaf = 50; p->max_per_target_leaf = 5; }
        else if (compute_type == CLUSTER_PARTICLE) { p->max_per_source_leaf = 5; p->max_per_target_leaf = 50; }
        else { p->max_per_source_leaf = 50; p->max_per_target_leaf = 50; }
    }
    RunParams_Validate(p);
}

void RunParams_Validate(struct RunParams *p)
{
    if (!p) return;
    const int m = p->interp_degree + 1;
    p->interp_pts_per_cluster = m * m * m;
    p->interp_weights_per_cluster = p->interp_pts_per_cluster;
    p->interp_charges_per_cluster = p->interp_pts_per_cluster;
    if (p->approximation == HERMITE) {
        p->interp_charges_per_cluster *= 8;
        if (p->singularity == SUBTRACTION) p->interp_weights_per_cluster *= 8;
    }
}

void RunParams_Free(struct RunParams **run_params_addr)
{
    if (!run_params_addr || !*run_params_addr) return;
    struct RunParams *p = *run_params_addr;
    if (p->num_kernel_params > 0) free(p->kernel_params);
    free(p);
    *run_params_addr = NULL;
}

void RunParams_Print(struct RunParams *p)
{
    if (!p) return;
    printf("[BaryTree]\n[BaryTree] RunParams struct has been set to the following:\n[BaryTree]\n");
    printf("[BaryTree]                     kernel = %d\n", p->kernel);
    printf("[BaryTree]          num_kernel_params = %d\n", p->num_kernel_params);
    printf("[BaryTree]              kernel_params = ");
    for (int i = 0; i < p->num_kernel_params; i++) printf("%f, ", p->kernel_params[i]);
    printf("\n");
    printf("[BaryTree]              approximation = %d\n", p->approximation);
    printf("[BaryTree]                singularity = %d\n", p->singularity);
    printf("[BaryTree]               compute_type = %d\n", p->compute_type);
    printf("[BaryTree]                      theta = %f\n", p->theta);
    printf("[BaryTree]              interp_degree = %d\n", p->interp_degree);
    printf("[BaryTree]     interp_pts_per_cluster = %d\n", p->interp_pts_per_cluster);
    printf("[BaryTree] interp_weights_per_cluster = %d\n", p->interp_weights_per_cluster);
    printf("[BaryTree] interp_charges_per_cluster = %d\n", p->interp_charges_per_cluster);
    printf("[BaryTree]        max_per_source_leaf = %d\n", p->max_per_source_leaf);
    printf("[BaryTree]        max_per_target_leaf = %d\n", p->max_per_target_leaf);
    printf("[BaryTree]          size_check_factor = %f\n", p->size_check_factor);
    printf("[BaryTree]                       beta = %f\n", p->beta);
    printf("[BaryTree]                  verbosity = %d\n", p->verbosity);
    printf("[BaryTree]\n");
}

/* Particles_Validate (src/particles/particles.c:157-228): the required arrays
 * must be set, and subtraction needs source weights. */
static int check_particles(const struct Particles *s, const struct Particles *t, const struct RunParams *p,
                           const char *who)
{
    if (!s || !t || !p) {
        fprintf(stderr, "[BaryTree] ERROR (%d): %s: NULL sources, targets or run parameters\n", BT_ERR_PARAM, who);
        return 0;
    }
    if (!s->x || !s->y || !s->z || !s->q || !t->x || !t->y || !t->z) {
        fprintf(stderr, "[BaryTree] ERROR (%d): %s: one or more required particle arrays is unset\n",
                BT_ERR_PARAM, who);
        return 0;
    }
    if (p->singularity == SUBTRACTION && !s->w) {
        fprintf(stderr, "[BaryTree] ERROR (%d): %s: singularity subtraction requires source weights\n",
                BT_ERR_PARAM, who);
        return 0;
    }
    return 1;
}

static double *scratch(int n)
{
    return malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
}

void treedriver(struct Particles *sources, struct Particles *targets, struct RunParams *run_params,
                double *potential, double *time_tree)
{
    if (time_tree) memset(time_tree, 0, 13 * sizeof(double));
    if (!check_particles(sources, targets, run_params, "treedriver")) return;
    RunParams_Validate(run_params);
    if (run_params->verbosity > 0) {
        printf("[BaryTree]\n[BaryTree] BaryTree has started.\n");
        RunParams_Print(run_params);
    }
    const int nt = targets->num;
    double *tmp = scratch(nt);
    if (!tmp) {
        fprintf(stderr, "[BaryTree] ERROR (%d): treedriver: host allocation failed\n", BT_ERR_PARAM);
        return;
    }
    bt_report rep;
    memset(&rep, 0, sizeof rep);
    /* The struct already holds the resolved parameters (the caller may have
     * edited them after RunParams_Setup), so beta is not applied again. */
    int rc = bt_eval_ex(nt, sources->num, targets->x, targets->y, targets->z, targets->q, sources->x, sources->y,
                        sources->z, sources->q, sources->w, tmp, run_params->kernel, run_params->num_kernel_params,
                        run_params->kernel_params, run_params->singularity, run_params->approximation,
                        run_params->compute_type, run_params->theta, run_params->interp_degree,
                        run_params->max_per_source_leaf, run_params->max_per_target_leaf,
                        run_params->size_check_factor, -1.0, NULL, &rep);
    if (rc != BT_OK) {
        fprintf(stderr, "[BaryTree] ERROR (%d): treedriver: %s\n", rc, bt_last_error());
        free(tmp);
        return;
    }
    for (int i = 0; i < nt; i++) potential[i] += tmp[i];
    free(tmp);
    if (time_tree) {
        time_tree[0] = rep.ms_setup * 1e-3;
        time_tree[2] = rep.ms_upward * 1e-3;
        time_tree[5] = rep.ms_compute * 1e-3;
        time_tree[8] = rep.ms_downward * 1e-3;
        time_tree[9] = rep.ms_transfer * 1e-3;
        time_tree[11] = time_tree[0];
        time_tree[12] = time_tree[5] + time_tree[8];
    }
    if (run_params->verbosity > 0) {
        printf("[BaryTree] Interactions: %lld PP, %lld PC, %lld CP, %lld CC (pointwise %lld, %lld, %lld, %lld)\n",
               rep.num_pp, rep.num_pc, rep.num_cp, rep.num_cc, rep.pp_ptwise, rep.pc_ptwise, rep.cp_ptwise,
               rep.cc_ptwise);
        printf("[BaryTree] BaryTree has finished.\n[BaryTree]\n");
    }
}

void directdriver(struct Particles *sources, struct Particles *targets, struct RunParams *run_params,
                  double *potential, double *time_direct)
{
    if (time_direct) memset(time_direct, 0, 4 * sizeof(double));
    if (!check_particles(sources, targets, run_params, "directdriver")) return;
    const int nt = targets->num;
    double *tmp = scratch(nt);
    if (!tmp) {
        fprintf(stderr, "[BaryTree] ERROR (%d): directdriver: host allocation failed\n", BT_ERR_PARAM);
        return;
    }
    const double t0 = wall_s();
    int rc = bt_direct_full(nt, sources->num, targets->x, targets->y, targets->z, targets->q, sources->x,
                            sources->y, sources->z, sources->q, sources->w, tmp, run_params->kernel,
                            run_params->num_kernel_params, run_params->kernel_params, run_params->singularity, 0);
    if (rc != BT_OK) {
        fprintf(stderr, "[BaryTree] ERROR (%d): directdriver: %s\n", rc, bt_last_error());
        free(tmp);
        return;
    }
    for (int i = 0; i < nt; i++) potential[i] += tmp[i];
    free(tmp);
    if (time_direct) time_direct[2] = wall_s() - t0;
}
