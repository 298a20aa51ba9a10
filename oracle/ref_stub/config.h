/* Build configuration for the reference library compiled as the GPU
 * reference baseline (test infrastructure only): the single-GPU entry points
 * of the reference are declared only under HAVE_MPI, which the single-rank
 * stub in mpi.h beside this file satisfies. */
#define HAVE_MPI 1
