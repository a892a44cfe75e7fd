/* MKL-compatibility shim (TEST INFRASTRUCTURE ONLY): the DFTI subset the reference uses —
 * one-dimensional real transforms of power-of-two length in double precision, out of place,
 * conjugate-even output stored as n/2 + 1 complex values (COMPLEX_COMPLEX), optionally batched
 * (NUMBER_OF_TRANSFORMS with INPUT/OUTPUT_DISTANCE in elements of each side's domain), with a
 * backward scale. Implemented in mkl_shim.c. */
#ifndef SSA_MKLSHIM_DFTI_H
#define SSA_MKLSHIM_DFTI_H

#include "mkl.h"

#ifdef __cplusplus
extern "C" {
#endif

enum DFTI_CONFIG_PARAM {
    DFTI_PLACEMENT = 11,
    DFTI_CONJUGATE_EVEN_STORAGE = 18,
    DFTI_NUMBER_OF_TRANSFORMS = 7,
    DFTI_INPUT_DISTANCE = 14,
    DFTI_OUTPUT_DISTANCE = 15,
    DFTI_FORWARD_SCALE = 4,
    DFTI_BACKWARD_SCALE = 5
};

enum DFTI_CONFIG_VALUE {
    DFTI_SINGLE = 35,
    DFTI_DOUBLE = 36,
    DFTI_COMPLEX = 32,
    DFTI_REAL = 33,
    DFTI_INPLACE = 43,
    DFTI_NOT_INPLACE = 44,
    DFTI_COMPLEX_COMPLEX = 39,
    DFTI_COMPLEX_REAL = 40
};

typedef struct ssa_shim_dfti *DFTI_DESCRIPTOR_HANDLE;

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *h, enum DFTI_CONFIG_VALUE precision,
                              enum DFTI_CONFIG_VALUE domain, MKL_LONG dimension, MKL_LONG length);
MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE h, enum DFTI_CONFIG_PARAM param, ...);
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE h);
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE h, void *in, ...);
MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE h, void *in, ...);
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *h);

#ifdef __cplusplus
}
#endif

#endif
