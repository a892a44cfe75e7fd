/* MKL-compatibility shim (TEST INFRASTRUCTURE ONLY): VML elementwise products as loops. */
#ifndef SSA_MKLSHIM_VML_H
#define SSA_MKLSHIM_VML_H

#include "mkl.h"

#ifdef __cplusplus
extern "C" {
#endif

void vzMul(MKL_INT n, const MKL_Complex16 *a, const MKL_Complex16 *b, MKL_Complex16 *r);
void vzMulByConj(MKL_INT n, const MKL_Complex16 *a, const MKL_Complex16 *b, MKL_Complex16 *r);
void vdMul(MKL_INT n, const double *a, const double *b, double *r);

#ifdef __cplusplus
}
#endif

#endif
