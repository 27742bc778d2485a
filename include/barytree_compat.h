/*
 * barytree_compat.h -- BaryTree's internal driver interface, served by
 * libbarytree_b200.so.
 *
 * Programs written against the reference's drivers rather than its public
 * entry point (its own test program, tests/serial_tests.c, calls treedriver
 * and directdriver with Particles and RunParams structs) link against this
 * library unchanged.  The two structs restate the reference's layouts field
 * for field (src/particles/struct_particles.h:5-27,
 * src/run_params/struct_run_params.h:7-31): the layout is the ABI, so the
 * include guards are the reference's too and either header set can be used.
 *
 * Differences from the reference, all on the safe side:
 *   - the particle arrays are only read (the reference permutes them in place
 *     and restores them on exit, src/drivers/treedriver.c:304-305);
 *   - invalid or unsupported runs print the reason and return without
 *     touching the potential (the reference calls exit);
 *   - RunParams_Free clears the caller's pointer.
 */
#ifndef BARYTREE_COMPAT_H
#define BARYTREE_COMPAT_H

#include "barytree_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifndef H_PARTICLES_H
#define H_PARTICLES_H
/* src/particles/struct_particles.h:5-27 */
struct Particles {
    int num;
    double *x, *y, *z, *q;
    double *w;                  /* quadrature weights (singularity subtraction) */
    int *ibeg, *iend;
    int *order;
    int sources_w_dummy, targets_q_dummy;
    int targets_x_duplicate, targets_y_duplicate, targets_z_duplicate, targets_q_duplicate;
};
#endif

#ifndef H_RUN_PARAMS_H
#define H_RUN_PARAMS_H
/* src/run_params/struct_run_params.h:7-31 */
struct RunParams {
    KERNEL kernel;
    int num_kernel_params;
    double *kernel_params;
    APPROXIMATION approximation;
    SINGULARITY singularity;
    COMPUTE_TYPE compute_type;
    double theta;
    double size_check_factor;
    int interp_degree;
    int interp_pts_per_cluster;
    int interp_charges_per_cluster;
    int interp_weights_per_cluster;
    int max_per_source_leaf;
    int max_per_target_leaf;
    double beta;
    int verbosity;
};
#endif

/* src/run_params/run_params.h:8-22 (run_params.c:13-131): allocates
 * *run_params_addr (freeing a previous one) and fills it; beta in [0,1]
 * derives theta, degree, size check and leaf sizes. */
void RunParams_Setup(struct RunParams **run_params_addr,
                     KERNEL kernel, int num_kernel_params, double *kernel_params,
                     APPROXIMATION approximation, SINGULARITY singularity, COMPUTE_TYPE compute_type,
                     double theta, int interp_degree,
                     int max_per_source_leaf, int max_per_target_leaf, double size_check_factor,
                     double beta, int verbosity);

/* run_params.c:135-148: recomputes the per-cluster counts from the degree,
 * approximation and singularity (callers may edit the struct after Setup). */
void RunParams_Validate(struct RunParams *run_params);

void RunParams_Free(struct RunParams **run_params_addr);

void RunParams_Print(struct RunParams *run_params);

/* src/drivers/treedriver.h:8-9.  Treecode potential of the sources at the
 * targets with the struct's parameters, ADDED to potential[] in the caller's
 * target order (the reference accumulates too; with a zeroed array the
 * results agree).  time_tree[0..12] receives phase times in seconds:
 * [0] tree and list setup, [2] upward pass, [5] evaluation, [8] downward
 * pass, [9] transfers and output ordering, [11] = setup, [12] = [5]+[8]. */
void treedriver(struct Particles *sources, struct Particles *targets, struct RunParams *run_params,
                double *potential, double *time_tree);

/* src/drivers/directdriver.h:8-9.  FP64 direct sum ADDED to potential[],
 * with the subtraction pair term and correction when the struct asks for
 * singularity subtraction.  time_direct[0..3]: [2] the sum, [3] 0. */
void directdriver(struct Particles *sources, struct Particles *targets, struct RunParams *run_params,
                  double *potential, double *time_direct);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* BARYTREE_COMPAT_H */
