/*
 * Build shim for compiling the reference's FP64 CPU core on Linux.
 *
 * The reference's QualityContactSolver.cpp includes Apple's Accelerate
 * framework for a single LAPACK routine, dsyev_ (symmetric eigenvalues,
 * JOBZ = 'N'), used only as a minimum-eigenvalue admission check.  This
 * header declares that one routine with 64-bit LAPACK integers; the
 * definition lives in oracle/shim/dsyev_jacobi.cpp (a cyclic Jacobi
 * eigenvalue method, written for this project).  Test infrastructure only.
 */
#pragma once

#include <stdint.h>

typedef int64_t __LAPACK_int;

#ifdef __cplusplus
extern "C" {
#endif

void dsyev_(
    const char* jobz,
    const char* uplo,
    const __LAPACK_int* n,
    double* a,
    const __LAPACK_int* lda,
    double* w,
    double* work,
    const __LAPACK_int* lwork,
    __LAPACK_int* info
);

#ifdef __cplusplus
}
#endif
