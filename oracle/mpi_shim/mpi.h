/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference
 * BaryTree C sources on a machine without an MPI installation.
 *
 * Test infrastructure: nothing in the barytree_b200 product includes this.
 *
 * Semantics: one rank (rank 0, size 1).  Collectives copy the send buffer to
 * the receive buffer, the barrier is a no-op, memory allocation is malloc,
 * and the one-sided window calls do nothing.  With one rank the reference
 * never enters its remote (locally-essential-tree) code paths
 * (src/drivers/treedriver.c:221,422,712 test num_procs > 1), so the window
 * calls are only compiled, never relied upon.
 */
#ifndef BT_ORACLE_MPI_SHIM_H
#define BT_ORACLE_MPI_SHIM_H

#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;   /* encodes the element size in bytes */
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Win;
typedef long MPI_Aint;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_SUCCESS 0
#define MPI_LOCK_SHARED 1
#define MPI_LOCK_EXCLUSIVE 2

#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_LONG_LONG_INT ((MPI_Datatype)sizeof(long long))
#define MPI_LONG_LONG MPI_LONG_LONG_INT

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }

static inline double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
    (void)op; (void)root; (void)c;
    if (s != r) memcpy(r, s, (size_t)n * (size_t)t);
    return 0;
}

static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    return MPI_Reduce(s, r, n, t, op, 0, c);
}

static inline int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{
    (void)rn; (void)rt; (void)c;
    if (s != r) memcpy(r, s, (size_t)sn * (size_t)st);
    return 0;
}

static inline int MPI_Alloc_mem(MPI_Aint size, MPI_Info info, void *baseptr)
{
    (void)info;
    *(void **)baseptr = malloc(size > 0 ? (size_t)size : 1);
    return 0;
}

static inline int MPI_Free_mem(void *p) { free(p); return 0; }

static inline int MPI_Win_create(void *b, MPI_Aint s, int d, MPI_Info i, MPI_Comm c, MPI_Win *w)
{ (void)b; (void)s; (void)d; (void)i; (void)c; *w = 0; return 0; }
static inline int MPI_Win_free(MPI_Win *w) { (void)w; return 0; }
static inline int MPI_Win_lock(int l, int r, int a, MPI_Win w) { (void)l; (void)r; (void)a; (void)w; return 0; }
static inline int MPI_Win_unlock(int r, MPI_Win w) { (void)r; (void)w; return 0; }
static inline int MPI_Get(void *o, int on, MPI_Datatype ot, int r, MPI_Aint d, int tn, MPI_Datatype tt, MPI_Win w)
{ (void)o; (void)on; (void)ot; (void)r; (void)d; (void)tn; (void)tt; (void)w; return 0; }

static inline int MPI_Type_create_indexed_block(int n, int bl, const int *d, MPI_Datatype o, MPI_Datatype *t)
{ (void)n; (void)bl; (void)d; *t = o; return 0; }
static inline int MPI_Type_indexed(int n, const int *bl, const int *d, MPI_Datatype o, MPI_Datatype *t)
{ (void)n; (void)bl; (void)d; *t = o; return 0; }
static inline int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
static inline int MPI_Type_free(MPI_Datatype *t) { (void)t; return 0; }

#endif /* BT_ORACLE_MPI_SHIM_H */
