/* MKL-compatibility shim (TEST INFRASTRUCTURE ONLY): the LAPACKE subset the reference's
 * double-precision build calls, bound to scipy's bundled OpenBLAS (LP64). */
#ifndef SSA_MKLSHIM_LAPACKE_H
#define SSA_MKLSHIM_LAPACKE_H

#include "mkl.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

lapack_int scipy_LAPACKE_dgeqrf(int layout, lapack_int m, lapack_int n, double *a, lapack_int lda,
                                double *tau);
lapack_int scipy_LAPACKE_dorgqr(int layout, lapack_int m, lapack_int n, lapack_int k, double *a,
                                lapack_int lda, const double *tau);
lapack_int scipy_LAPACKE_dgesdd_work(int layout, char jobz, lapack_int m, lapack_int n, double *a,
                                     lapack_int lda, double *s, double *u, lapack_int ldu,
                                     double *vt, lapack_int ldvt, double *work, lapack_int lwork,
                                     lapack_int *iwork);
lapack_int scipy_LAPACKE_dgesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n,
                                double *a, lapack_int lda, double *s, double *u, lapack_int ldu,
                                double *vt, lapack_int ldvt, double *superb);
lapack_int scipy_LAPACKE_dgels_work(int layout, char trans, lapack_int m, lapack_int n,
                                    lapack_int nrhs, double *a, lapack_int lda, double *b,
                                    lapack_int ldb, double *work, lapack_int lwork);
lapack_int scipy_LAPACKE_dgeev(int layout, char jobvl, char jobvr, lapack_int n, double *a,
                               lapack_int lda, double *wr, double *wi, double *vl,
                               lapack_int ldvl, double *vr, lapack_int ldvr);

#define LAPACKE_dgeqrf scipy_LAPACKE_dgeqrf
#define LAPACKE_dorgqr scipy_LAPACKE_dorgqr
#define LAPACKE_dgesdd_work scipy_LAPACKE_dgesdd_work
#define LAPACKE_dgesvd scipy_LAPACKE_dgesvd
#define LAPACKE_dgels_work scipy_LAPACKE_dgels_work
#define LAPACKE_dgeev scipy_LAPACKE_dgeev

#ifdef __cplusplus
}
#endif

#endif
