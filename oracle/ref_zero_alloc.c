/*
 * ref_zero_alloc.c -- zero-initialising replacement for the reference's
 * malloc_or_exit (src/utilities/xmalloc.c:17), linked into the reference
 * oracle build in place of that file.
 *
 * Why: on the reference's CPU path, Clusters_Targets_Construct allocates the
 * target-grid potentials with make_vector (src/clusters/clusters.c:234) and
 * zeroes them only inside the OpenACC branch (:242-256).  The CPU build then
 * accumulates CP/CC results onto uninitialised heap memory and returns
 * garbage or NaN whenever the allocator recycles memory.  Zero-filling every
 * allocation reproduces the OpenACC path's explicit zeroing and changes
 * nothing else (every other array the reference allocates is written before
 * it is read).  Same failure behaviour as the original: exit on failure or on
 * a zero-byte request.
 */
#include <stdio.h>
#include <stdlib.h>

void *malloc_or_exit(size_t nbytes, const char *file, int line)
{
    void *x;
    if (nbytes == 0 || (x = calloc(1, nbytes)) == NULL) {
        fprintf(stderr, "%s: line %d: malloc() of %zu bytes failed\n", file, line, nbytes);
        exit(EXIT_FAILURE);
    }
    return x;
}
