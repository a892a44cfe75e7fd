/* MKL-compatibility shim (TEST INFRASTRUCTURE ONLY): declarations that let the reference's
 * unmodified MKL/ssa_opt.h compile and run without Intel MKL, which is absent here.
 *
 * What stands in for what:
 *   CBLAS / LAPACKE  -> scipy's bundled OpenBLAS (LP64 symbols scipy_cblas_* / scipy_LAPACKE_*),
 *                       bound by the macros in this header and mkl_lapacke.h;
 *   DFTI             -> our own real FFT (mkl_shim.c: Stockham radix-4/2 on the half-length
 *                       complex sequence + real pre/post-processing), power-of-two lengths;
 *   VML              -> plain loops (complex / real elementwise products);
 *   VSL              -> draws read from a host-registered buffer (each new stream starts at its
 *                       beginning, as a fresh MKL stream with the same seed restarts its
 *                       sequence), or a counter-based generator when none is registered;
 *   mkl_malloc/free  -> aligned_alloc / free.
 * Only the subset the reference's double-precision build uses is provided. */
#ifndef SSA_MKLSHIM_MKL_H
#define SSA_MKLSHIM_MKL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef long MKL_LONG;
typedef int MKL_INT;
typedef struct { double real, imag; } MKL_Complex16;
typedef struct { float real, imag; } MKL_Complex8;

void *mkl_malloc(size_t size, int alignment);
void mkl_free(void *p);
void mkl_set_num_threads(int n);
int mkl_get_max_threads(void);

/* CBLAS: standard enumerator values (shared by every CBLAS, OpenBLAS included). */
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;

double scipy_cblas_ddot(int n, const double *x, int incx, const double *y, int incy);
double scipy_cblas_dnrm2(int n, const double *x, int incx);
void scipy_cblas_dscal(int n, double a, double *x, int incx);
void scipy_cblas_daxpy(int n, double a, const double *x, int incx, double *y, int incy);
void scipy_cblas_dcopy(int n, const double *x, int incx, double *y, int incy);
void scipy_cblas_dswap(int n, double *x, int incx, double *y, int incy);
void scipy_cblas_dgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE trans, int m, int n, double alpha,
                       const double *a, int lda, const double *x, int incx, double beta, double *y,
                       int incy);
void scipy_cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int m, int n,
                       int k, double alpha, const double *a, int lda, const double *b, int ldb,
                       double beta, double *c, int ldc);
void scipy_cblas_dsyrk(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans, int n, int k,
                       double alpha, const double *a, int lda, double beta, double *c, int ldc);

#define cblas_ddot scipy_cblas_ddot
#define cblas_dnrm2 scipy_cblas_dnrm2
#define cblas_dscal scipy_cblas_dscal
#define cblas_daxpy scipy_cblas_daxpy
#define cblas_dcopy scipy_cblas_dcopy
#define cblas_dswap scipy_cblas_dswap
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_dsyrk scipy_cblas_dsyrk

#ifdef __cplusplus
}
#endif

#endif
