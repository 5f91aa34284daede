/*
 * Minimal BLAS level-1 routines for linking the reference bml sources into
 * the oracle library (oracle/_ref/libbml_ref.so).  Test infrastructure only.
 *
 * The reference calls ?scal / ?axpy through the C_SSCAL/C_DSCAL/... macros
 * (src/C-interface/blas.h:8-17, used by ellpack/bml_scale_ellpack_typed.c:85,119).
 * Dense GEMM goes through its internal GEMM when BML_INTERNAL_GEMM is defined
 * (src/internal-blas/bml_gemm.c), so only level-1 kernels are needed here.
 * Each routine is the textbook definition (x <- a*x, y <- a*x + y) with one
 * correctly rounded multiply (and add) per element, which is what any BLAS
 * produces for these operations on finite inputs.
 */
void oracle_sscal_(const int *n, const float *a, float *x, const int *incx)
{
    for (int i = 0; i < *n; i++)
        x[(long) i * *incx] = *a * x[(long) i * *incx];
}

void oracle_dscal_(const int *n, const double *a, double *x, const int *incx)
{
    for (int i = 0; i < *n; i++)
        x[(long) i * *incx] = *a * x[(long) i * *incx];
}

void oracle_saxpy_(const int *n, const float *a, const float *x,
                   const int *incx, float *y, const int *incy)
{
    for (int i = 0; i < *n; i++)
        y[(long) i * *incy] = *a * x[(long) i * *incx] + y[(long) i * *incy];
}

void oracle_daxpy_(const int *n, const double *a, const double *x,
                   const int *incx, double *y, const int *incy)
{
    for (int i = 0; i < *n; i++)
        y[(long) i * *incy] = *a * x[(long) i * *incx] + y[(long) i * *incy];
}

/*
 * LAPACK entry points referenced (but, with HAVE_LAPACK undefined, never
 * reached on the multiply/add/threshold/trace/transpose path) by the
 * reference's dense diagonalize/inverse code.  They exist only so that the
 * library loads with immediate binding; calling one aborts.
 */
#include <stdio.h>
#include <stdlib.h>
#define ORACLE_LAPACK_STUB(name) \
    void name(void) { fprintf(stderr, "oracle: LAPACK %s not linked\n", #name); abort(); }
ORACLE_LAPACK_STUB(C_CHEEVR)
ORACLE_LAPACK_STUB(C_ZHEEVR)
ORACLE_LAPACK_STUB(C_SSYEV)
ORACLE_LAPACK_STUB(C_DSYEV)
ORACLE_LAPACK_STUB(C_SGETRF)
ORACLE_LAPACK_STUB(C_DGETRF)
ORACLE_LAPACK_STUB(C_SGETRI)
ORACLE_LAPACK_STUB(C_DGETRI)
