/* MKL-compatibility shim (TEST INFRASTRUCTURE ONLY): VSL streams whose Gaussian and uniform
 * draws come from host-registered buffers (mklshim_set_gaussian / mklshim_set_uniform in
 * mkl_shim.c). Every stream created after a registration reads that buffer from its start with
 * its own cursor — a fresh stream restarts the sequence, as a fresh MKL stream with the same
 * basic generator and seed does. Past the end of a buffer (or with none registered) the draws
 * come from a counter-based generator keyed by (seed, draw index); mklshim_draws_exhausted()
 * reports that this happened. */
#ifndef SSA_MKLSHIM_VSL_H
#define SSA_MKLSHIM_VSL_H

#include "mkl.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef void *VSLStreamStatePtr;

#define VSL_STATUS_OK 0
#define VSL_BRNG_MT19937 (1 << 20)
#define VSL_BRNG_MT2203 (2 << 20)
#define VSL_RNG_METHOD_GAUSSIAN_BOXMULLER 0
#define VSL_RNG_METHOD_GAUSSIAN_ICDF 2
#define VSL_RNG_METHOD_UNIFORM_STD 0

int vslNewStream(VSLStreamStatePtr *stream, MKL_INT brng, MKL_INT seed);
int vslDeleteStream(VSLStreamStatePtr *stream);
int vdRngGaussian(MKL_INT method, VSLStreamStatePtr stream, MKL_INT n, double *r, double a,
                  double sigma);
int vdRngUniform(MKL_INT method, VSLStreamStatePtr stream, MKL_INT n, double *r, double a,
                 double b);

#ifdef __cplusplus
}
#endif

#endif
