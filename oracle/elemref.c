/*
 * CPU oracle for the factor-and-solve path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of Elemental's sequential Cholesky / LU / solve
 * algorithms (file:line citations on every routine in oref_impl.h).  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
 * library, and only as the checker; the GPU product never calls it.
 *
 * Parity: pinned to the reference's own code (see oref_impl.h header).  Built by oracle/Makefile into
 * oracle/liboracle.so; exported names: oref_d* (double) and oref_s* (float).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define REAL double
#define PFX d
#include "oref_impl.h"
#undef REAL
#undef PFX

#define REAL float
#define PFX s
#include "oref_impl.h"
#undef REAL
#undef PFX

/* Thread count used by the OpenMP loops (0 = library default). */
#ifdef _OPENMP
#include <omp.h>
void oref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int oref_get_threads(void) { return omp_get_max_threads(); }
#else
void oref_set_threads(int n) { (void)n; }
int oref_get_threads(void) { return 1; }
#endif
