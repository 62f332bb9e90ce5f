/*
 * Build configuration of the reference's sources when they are compiled as
 * the CPU oracle (TEST INFRASTRUCTURE ONLY; oracle/refbuild/Makefile).  The
 * reference's CMake build would generate this file from its
 * cmake/config.h.cmake; this hand-written copy sets the few switches the
 * single-process oracle build needs: release mode (no call-stack tracing or
 * debug-only checks), Fortran BLAS/LAPACK names with a trailing underscore,
 * and an MPI that has MPI_IN_PLACE and MPI_Reduce_scatter_block.  No OpenMP,
 * Qt, PMRRR, FLAME or Fortran interface.
 */
#ifndef ELEMENTAL_CONFIG_H
#define ELEMENTAL_CONFIG_H 1

#define CMAKE_BUILD_TYPE PureRelease
#define Elemental_VERSION_MAJOR 0
#define Elemental_VERSION_MINOR 81

#define RESTRICT __restrict__
#define RELEASE
#define BLAS_POST
#define LAPACK_POST
#define HAVE_MPI_REDUCE_SCATTER_BLOCK
#define HAVE_MPI_IN_PLACE
#define HAVE_MPI_COMM_SET_ERRHANDLER
#define HAVE_MPI_INIT_THREAD
#define HAVE_MPI_QUERY_THREAD

#endif /* ELEMENTAL_CONFIG_H */
