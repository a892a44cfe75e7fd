/* MKL-compatibility shim (TEST INFRASTRUCTURE ONLY): implementations behind the declaration
 * headers in this directory, so that the reference's unmodified MKL/ssa_opt.h builds and runs
 * as a CPU checker and CPU baseline without Intel MKL.
 *
 * DFTI: a real transform of power-of-two length n is computed from the complex transform of
 * the h = n/2 point sequence z[j] = x[2j] + i x[2j+1] (the standard "two real halves" packing),
 * followed by the split into even/odd spectra and one twiddle per bin; the inverse runs the same
 * steps backwards. The h-point complex transform is a Stockham autosort FFT (Van Loan,
 * "Computational Frameworks for the Fast Fourier Transform", 1992, §1.7) with radix-4
 * decimation-in-frequency passes and one radix-2 pass when log2(h) is odd; twiddles are one
 * table W_h^t computed in double precision with libm at commit time. Semantics follow the
 * reference's use (MKL/ssa_opt.h:1111-1196, 2288-2311): out-of-place, conjugate-even output in
 * n/2 + 1 complex values, batches via NUMBER_OF_TRANSFORMS with INPUT/OUTPUT_DISTANCE counted in
 * elements of each side's domain, forward unscaled, backward multiplied by BACKWARD_SCALE.
 *
 * VSL: see mkl_vsl.h. VML: elementwise loops (aliasing of output and input allowed). */
#define _GNU_SOURCE
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mkl.h"
#include "mkl_dfti.h"
#include "mkl_vml.h"
#include "mkl_vsl.h"

#define SHIM_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------------------------ */
/* memory                                                                                      */
/* ------------------------------------------------------------------------------------------ */

void *mkl_malloc(size_t size, int alignment)
{
    if (alignment < 64)
        alignment = 64;
    size_t sz = (size + (size_t)alignment - 1) / (size_t)alignment * (size_t)alignment;
    return aligned_alloc((size_t)alignment, sz ? sz : (size_t)alignment);
}

void mkl_free(void *p) { free(p); }
void mkl_set_num_threads(int n) { (void)n; }
int mkl_get_max_threads(void) { return 1; }

/* ------------------------------------------------------------------------------------------ */
/* complex FFT core                                                                            */
/* ------------------------------------------------------------------------------------------ */

typedef struct { double re, im; } cpx;

/* One Stockham DIF pass family over h points: x (input) and y (scratch) alternate; returns the
 * buffer holding the result. tw[t] = exp(-2 pi i t / h), t < h. sign = -1 forward, +1 inverse
 * (conjugated twiddles and rotation). */
static cpx *stockham(int h, cpx *x, cpx *y, const cpx *tw, int sign)
{
    int n = h, s = 1;
    while (n >= 4) {
        const int n1 = n / 4;
        const int tstride = s; /* W_n^p = W_h^{p s} */
        for (int p = 0; p < n1; p++) {
            cpx w1 = tw[(size_t)p * tstride];
            cpx w2 = tw[(size_t)2 * p * tstride];
            cpx w3 = tw[(size_t)3 * p * tstride];
            if (sign > 0) {
                w1.im = -w1.im;
                w2.im = -w2.im;
                w3.im = -w3.im;
            }
            const cpx *xa = x + (size_t)s * p;
            const cpx *xb = x + (size_t)s * (p + n1);
            const cpx *xc = x + (size_t)s * (p + 2 * n1);
            const cpx *xd = x + (size_t)s * (p + 3 * n1);
            cpx *y0 = y + (size_t)s * (4 * p + 0);
            cpx *y1 = y + (size_t)s * (4 * p + 1);
            cpx *y2 = y + (size_t)s * (4 * p + 2);
            cpx *y3 = y + (size_t)s * (4 * p + 3);
            for (int q = 0; q < s; q++) {
                const double apc_r = xa[q].re + xc[q].re, apc_i = xa[q].im + xc[q].im;
                const double amc_r = xa[q].re - xc[q].re, amc_i = xa[q].im - xc[q].im;
                const double bpd_r = xb[q].re + xd[q].re, bpd_i = xb[q].im + xd[q].im;
                /* j (b - d) for the forward transform (rotation by -i of the DIF butterfly is
                 * expressed as +/- i depending on the direction) */
                double bmd_r = xb[q].re - xd[q].re, bmd_i = xb[q].im - xd[q].im;
                double jr, ji; /* rot = -i*sign_fwd*(b-d): forward uses -i, inverse +i */
                if (sign < 0) {
                    jr = bmd_i;
                    ji = -bmd_r;
                } else {
                    jr = -bmd_i;
                    ji = bmd_r;
                }
                y0[q].re = apc_r + bpd_r;
                y0[q].im = apc_i + bpd_i;
                const double t1r = amc_r + jr, t1i = amc_i + ji;
                const double t2r = apc_r - bpd_r, t2i = apc_i - bpd_i;
                const double t3r = amc_r - jr, t3i = amc_i - ji;
                y1[q].re = t1r * w1.re - t1i * w1.im;
                y1[q].im = t1r * w1.im + t1i * w1.re;
                y2[q].re = t2r * w2.re - t2i * w2.im;
                y2[q].im = t2r * w2.im + t2i * w2.re;
                y3[q].re = t3r * w3.re - t3i * w3.im;
                y3[q].im = t3r * w3.im + t3i * w3.re;
            }
        }
        cpx *t = x;
        x = y;
        y = t;
        n /= 4;
        s *= 4;
    }
    if (n == 2) {
        const cpx *xa = x, *xb = x + s;
        cpx *y0 = y, *y1 = y + s;
        for (int q = 0; q < s; q++) {
            const cpx a = xa[q], b = xb[q];
            y0[q].re = a.re + b.re;
            y0[q].im = a.im + b.im;
            y1[q].re = a.re - b.re;
            y1[q].im = a.im - b.im;
        }
        return y;
    }
    return x;
}

/* ------------------------------------------------------------------------------------------ */
/* DFTI descriptors                                                                            */
/* ------------------------------------------------------------------------------------------ */

struct ssa_shim_dfti {
    int n, h;
    int committed;
    long ntrans, idist, odist;
    int idist_set, odist_set;
    double fscale, bscale;
    cpx *tw;   /* W_h^t, t < h */
    cpx *rtw;  /* W_n^k, k <= h */
    cpx *buf0, *buf1;
};

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *hp, enum DFTI_CONFIG_VALUE precision,
                              enum DFTI_CONFIG_VALUE domain, MKL_LONG dimension, MKL_LONG length)
{
    if (!hp)
        return 1;
    *hp = NULL;
    if (precision != DFTI_DOUBLE || domain != DFTI_REAL || dimension != 1 || length < 2 ||
        (length & (length - 1)))
        return 1;
    struct ssa_shim_dfti *d = calloc(1, sizeof(*d));
    if (!d)
        return 1;
    d->n = (int)length;
    d->h = (int)length / 2;
    d->ntrans = 1;
    d->fscale = 1.0;
    d->bscale = 1.0;
    *hp = d;
    return 0;
}

MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE d, enum DFTI_CONFIG_PARAM param, ...)
{
    if (!d)
        return 1;
    va_list ap;
    va_start(ap, param);
    MKL_LONG rc = 0;
    switch (param) {
    case DFTI_PLACEMENT: {
        int v = va_arg(ap, int);
        rc = (v == DFTI_NOT_INPLACE) ? 0 : 1;
        break;
    }
    case DFTI_CONJUGATE_EVEN_STORAGE: {
        int v = va_arg(ap, int);
        rc = (v == DFTI_COMPLEX_COMPLEX) ? 0 : 1;
        break;
    }
    case DFTI_NUMBER_OF_TRANSFORMS:
        d->ntrans = va_arg(ap, MKL_LONG);
        rc = d->ntrans >= 1 ? 0 : 1;
        break;
    case DFTI_INPUT_DISTANCE:
        d->idist = va_arg(ap, MKL_LONG);
        d->idist_set = 1;
        break;
    case DFTI_OUTPUT_DISTANCE:
        d->odist = va_arg(ap, MKL_LONG);
        d->odist_set = 1;
        break;
    case DFTI_FORWARD_SCALE:
        d->fscale = va_arg(ap, double);
        break;
    case DFTI_BACKWARD_SCALE:
        d->bscale = va_arg(ap, double);
        break;
    default:
        rc = 1;
    }
    va_end(ap);
    d->committed = 0;
    return rc;
}

MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE d)
{
    if (!d)
        return 1;
    const int h = d->h, n = d->n;
    if (!d->tw) {
        d->tw = malloc(sizeof(cpx) * (size_t)(h > 0 ? h : 1));
        d->rtw = malloc(sizeof(cpx) * (size_t)(h + 1));
        d->buf0 = malloc(sizeof(cpx) * (size_t)(h > 0 ? h : 1));
        d->buf1 = malloc(sizeof(cpx) * (size_t)(h > 0 ? h : 1));
        if (!d->tw || !d->rtw || !d->buf0 || !d->buf1)
            return 1;
        for (int t = 0; t < h; t++) {
            const double a = -2.0 * M_PI * (double)t / (double)h;
            d->tw[t].re = cos(a);
            d->tw[t].im = sin(a);
        }
        for (int k = 0; k <= h; k++) {
            const double a = -2.0 * M_PI * (double)k / (double)n;
            d->rtw[k].re = cos(a);
            d->rtw[k].im = sin(a);
        }
    }
    d->committed = 1;
    return 0;
}

MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *hp)
{
    if (!hp || !*hp)
        return 0;
    struct ssa_shim_dfti *d = *hp;
    free(d->tw);
    free(d->rtw);
    free(d->buf0);
    free(d->buf1);
    free(d);
    *hp = NULL;
    return 0;
}

/* one real forward transform: x[n] -> X[h + 1] complex */
static void real_forward(struct ssa_shim_dfti *d, const double *x, cpx *X)
{
    const int h = d->h;
    cpx *z = d->buf0;
    for (int j = 0; j < h; j++) {
        z[j].re = x[2 * j];
        z[j].im = x[2 * j + 1];
    }
    const cpx *Z = stockham(h, z, d->buf1, d->tw, -1);
    for (int k = 0; k <= h; k++) {
        const cpx a = Z[k == h ? 0 : k];
        const cpx b = Z[(h - k) % h]; /* conj taken below */
        /* E = (a + conj b) / 2 ; O = (a - conj b) / (2i) */
        const double er = 0.5 * (a.re + b.re), ei = 0.5 * (a.im - b.im);
        const double dr = 0.5 * (a.re - b.re), di = 0.5 * (a.im + b.im);
        /* (dr + i di) / i = di - i dr */
        const double orr = di, oi = -dr;
        const cpx w = d->rtw[k];
        X[k].re = d->fscale * (er + (orr * w.re - oi * w.im));
        X[k].im = d->fscale * (ei + (orr * w.im + oi * w.re));
    }
}

/* one real backward transform: X[h + 1] complex -> x[n], scaled by bscale */
static void real_backward(struct ssa_shim_dfti *d, const cpx *X, double *x)
{
    const int h = d->h;
    cpx *Zb = d->buf0;
    for (int k = 0; k < h; k++) {
        cpx a = X[k], b = X[h - k];
        if (k == 0) {
            a.im = 0.0;
            b.im = 0.0;
        }
        /* E = (a + conj b)/2 ; O = (a - conj b) * conj(W_n^k) / 2 ; Z = E + i O */
        const double er = 0.5 * (a.re + b.re), ei = 0.5 * (a.im - b.im);
        const double tr = 0.5 * (a.re - b.re), ti = 0.5 * (a.im + b.im);
        const cpx w = d->rtw[k];
        const double orr = tr * w.re + ti * w.im;  /* t * conj(w) */
        const double oi = ti * w.re - tr * w.im;
        Zb[k].re = er - oi;
        Zb[k].im = ei + orr;
    }
    const cpx *z = stockham(h, Zb, d->buf1, d->tw, +1);
    const double s = 2.0 * d->bscale;
    for (int j = 0; j < h; j++) {
        x[2 * j] = s * z[j].re;
        x[2 * j + 1] = s * z[j].im;
    }
}

MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE d, void *in, ...)
{
    if (!d || !d->committed)
        return 1;
    va_list ap;
    va_start(ap, in);
    void *out = va_arg(ap, void *);
    va_end(ap);
    const long idist = d->idist_set ? d->idist : d->n;
    const long odist = d->odist_set ? d->odist : d->h + 1;
    for (long t = 0; t < d->ntrans; t++)
        real_forward(d, (const double *)in + t * idist, (cpx *)out + t * odist);
    return 0;
}

MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE d, void *in, ...)
{
    if (!d || !d->committed)
        return 1;
    va_list ap;
    va_start(ap, in);
    void *out = va_arg(ap, void *);
    va_end(ap);
    const long idist = d->idist_set ? d->idist : d->h + 1;
    const long odist = d->odist_set ? d->odist : d->n;
    for (long t = 0; t < d->ntrans; t++)
        real_backward(d, (const cpx *)in + t * idist, (double *)out + t * odist);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* VML                                                                                         */
/* ------------------------------------------------------------------------------------------ */

void vzMul(MKL_INT n, const MKL_Complex16 *a, const MKL_Complex16 *b, MKL_Complex16 *r)
{
    for (MKL_INT i = 0; i < n; i++) {
        const double ar = a[i].real, ai = a[i].imag, br = b[i].real, bi = b[i].imag;
        r[i].real = ar * br - ai * bi;
        r[i].imag = ar * bi + ai * br;
    }
}

void vzMulByConj(MKL_INT n, const MKL_Complex16 *a, const MKL_Complex16 *b, MKL_Complex16 *r)
{
    for (MKL_INT i = 0; i < n; i++) {
        const double ar = a[i].real, ai = a[i].imag, br = b[i].real, bi = b[i].imag;
        r[i].real = ar * br + ai * bi;
        r[i].imag = ai * br - ar * bi;
    }
}

void vdMul(MKL_INT n, const double *a, const double *b, double *r)
{
    for (MKL_INT i = 0; i < n; i++)
        r[i] = a[i] * b[i];
}

/* ------------------------------------------------------------------------------------------ */
/* VSL                                                                                         */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    uint64_t seed;
    long gpos, upos;      /* cursors into the registered buffers */
    uint64_t gctr, uctr;  /* counters of the fallback generator */
} shim_stream;

static const double *g_gauss;
static long g_gauss_n;
static const double *g_unif;
static long g_unif_n;
static int g_exhausted;

SHIM_EXPORT void mklshim_set_gaussian(const double *buf, long n)
{
    g_gauss = buf;
    g_gauss_n = buf ? n : 0;
    g_exhausted = 0;
}

SHIM_EXPORT void mklshim_set_uniform(const double *buf, long n)
{
    g_unif = buf;
    g_unif_n = buf ? n : 0;
    g_exhausted = 0;
}

SHIM_EXPORT int mklshim_draws_exhausted(void) { return g_exhausted; }

/* SplitMix64 finaliser (Steele, Lea, Flood, OOPSLA 2014) as a counter-based hash */
static uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double unit_open(uint64_t r) { return ((double)(r >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

int vslNewStream(VSLStreamStatePtr *stream, MKL_INT brng, MKL_INT seed)
{
    (void)brng;
    shim_stream *s = calloc(1, sizeof(*s));
    if (!s)
        return -1;
    s->seed = (uint64_t)(uint32_t)seed;
    *stream = s;
    return VSL_STATUS_OK;
}

int vslDeleteStream(VSLStreamStatePtr *stream)
{
    if (stream && *stream) {
        free(*stream);
        *stream = NULL;
    }
    return VSL_STATUS_OK;
}

int vdRngGaussian(MKL_INT method, VSLStreamStatePtr stream, MKL_INT n, double *r, double a,
                  double sigma)
{
    (void)method;
    shim_stream *s = stream;
    for (MKL_INT i = 0; i < n; i++) {
        double z;
        if (s->gpos < g_gauss_n) {
            z = g_gauss[s->gpos++];
        } else {
            if (g_gauss)
                g_exhausted = 1;
            const uint64_t c = s->gctr++;
            const uint64_t base = mix64(s->seed * 0x2545F4914F6CDD1Dull + (c >> 1));
            const double u1 = unit_open(mix64(base ^ 0x1111ull)), u2 = unit_open(mix64(base ^ 0x2222ull));
            const double rad = sqrt(-2.0 * log(u1));
            z = (c & 1) ? rad * sin(2.0 * M_PI * u2) : rad * cos(2.0 * M_PI * u2);
        }
        r[i] = a + sigma * z;
    }
    return VSL_STATUS_OK;
}

int vdRngUniform(MKL_INT method, VSLStreamStatePtr stream, MKL_INT n, double *r, double a, double b)
{
    (void)method;
    shim_stream *s = stream;
    for (MKL_INT i = 0; i < n; i++) {
        double u;
        if (s->upos < g_unif_n) {
            u = g_unif[s->upos++];
        } else {
            if (g_unif)
                g_exhausted = 1;
            u = unit_open(mix64(s->seed * 0x9E3779B97F4A7C15ull + 0x5555ull + s->uctr++));
        }
        r[i] = a + (b - a) * u;
    }
    return VSL_STATUS_OK;
}
