/* Build configuration for compiling the reference's CPU lmp sources as the
 * oracle's pin: OpenMP on, no MPI, no GPU, no vendor BLAS. */
#define WITH_OPENMP 1
