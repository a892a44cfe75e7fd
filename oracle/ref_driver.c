/*
 * Test-infrastructure driver around the reference's dependency-free C implementation
 * (MKL/ssa_opt_ref.h of SSA-Opt). It is compiled from the reference source where it lies by
 * oracle/Makefile into oracle/_ref/libssa_ref.so and is loaded ONLY by tests and by the CPU
 * baseline leg of bench.py, to pin the NumPy oracle and to time the reference CPU path.
 *
 * The driver adds flat entry points (plain pointers, ctypes friendly):
 *   - refdrv_omega: the Omega the reference's randomized SVD draws (xorshift64 + Box-Muller,
 *     ssa_opt_ref.h:305-327, drawn in order at ssa_opt_ref.h:1110-1111) from a given state;
 *   - refdrv_randomized: ssa_opt_ref_decompose_randomized (ssa_opt_ref.h:1063-1191);
 *   - refdrv_matvec / refdrv_matvec_T: the reference's Hankel matvecs (ssa_opt_ref.h:734-797);
 *   - refdrv_reconstruct / refdrv_wcorr / refdrv_lrf / refdrv_forecast on given factors;
 *   - refdrv_pipeline: init + randomized decompose + reconstruct groups + W-correlation, the
 *     reference CPU path timed as the baseline.
 */
#define SSA_OPT_REF_IMPLEMENTATION
#include "ssa_opt_ref.h"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define REFDRV_API __attribute__((visibility("default")))

REFDRV_API int refdrv_sizeof_ctx(void) { return (int)sizeof(SSA_Opt_Ref); }

REFDRV_API void refdrv_omega(uint64_t state, int K, int kp, double *omega)
{
    for (long i = 0; i < (long)K * kp; i++)
        omega[i] = ssa_ref_randn(&state);
}

REFDRV_API uint64_t refdrv_default_state(void)
{
    SSA_Opt_Ref s;
    double x[8] = {1, 2, 3, 4, 5, 6, 7, 8};
    memset(&s, 0, sizeof(s));
    if (ssa_opt_ref_init(&s, x, 8, 4) != 0)
        return 0;
    uint64_t st = s.rng_state;
    ssa_opt_ref_free(&s);
    return st;
}

REFDRV_API int refdrv_matvec(const double *x, int N, int L, const double *v, double *y)
{
    SSA_Opt_Ref s;
    memset(&s, 0, sizeof(s));
    if (ssa_opt_ref_init(&s, x, N, L) != 0)
        return -1;
    ssa_ref_hankel_matvec(&s, v, y);
    ssa_opt_ref_free(&s);
    return 0;
}

REFDRV_API int refdrv_matvec_T(const double *x, int N, int L, const double *u, double *z)
{
    SSA_Opt_Ref s;
    memset(&s, 0, sizeof(s));
    if (ssa_opt_ref_init(&s, x, N, L) != 0)
        return -1;
    ssa_ref_hankel_matvec_T(&s, u, z);
    ssa_opt_ref_free(&s);
    return 0;
}

/* Randomized decomposition with the rng state set to `state` first; writes U (L x k),
 * V (K x k), sigma (k). Returns the number of components or -1. */
REFDRV_API int refdrv_randomized(const double *x, int N, int L, int k, int p, uint64_t state,
                                 double *U, double *V, double *sigma)
{
    SSA_Opt_Ref s;
    memset(&s, 0, sizeof(s));
    if (ssa_opt_ref_init(&s, x, N, L) != 0)
        return -1;
    s.rng_state = state;
    if (ssa_opt_ref_decompose_randomized(&s, k, p) != 0)
    {
        ssa_opt_ref_free(&s);
        return -1;
    }
    int kk = s.n_components;
    memcpy(U, s.U, sizeof(double) * (size_t)L * kk);
    memcpy(V, s.V, sizeof(double) * (size_t)s.K * kk);
    memcpy(sigma, s.sigma, sizeof(double) * kk);
    ssa_opt_ref_free(&s);
    return kk;
}

/* Sequential power-iteration decomposition (ssa_opt_ref.h:859-1061). */
REFDRV_API int refdrv_sequential(const double *x, int N, int L, int k, int max_iter,
                                 double *U, double *V, double *sigma)
{
    SSA_Opt_Ref s;
    memset(&s, 0, sizeof(s));
    if (ssa_opt_ref_init(&s, x, N, L) != 0)
        return -1;
    if (ssa_opt_ref_decompose(&s, k, max_iter) != 0)
    {
        ssa_opt_ref_free(&s);
        return -1;
    }
    int kk = s.n_components;
    memcpy(U, s.U, sizeof(double) * (size_t)L * kk);
    memcpy(V, s.V, sizeof(double) * (size_t)s.K * kk);
    memcpy(sigma, s.sigma, sizeof(double) * kk);
    ssa_opt_ref_free(&s);
    return kk;
}

/* Context with the given factors installed as a finished decomposition. */
static int refdrv_ctx_with(SSA_Opt_Ref *s, const double *x, int N, int L, int k,
                           const double *U, const double *V, const double *sigma)
{
    memset(s, 0, sizeof(*s));
    if (ssa_opt_ref_init(s, x, N, L) != 0)
        return -1;
    int K = s->K;
    s->U = (double *)ssa_ref_alloc(sizeof(double) * (size_t)L * k);
    s->V = (double *)ssa_ref_alloc(sizeof(double) * (size_t)K * k);
    s->sigma = (double *)ssa_ref_alloc(sizeof(double) * k);
    s->eigenvalues = (double *)ssa_ref_alloc(sizeof(double) * k);
    if (!s->U || !s->V || !s->sigma || !s->eigenvalues)
    {
        ssa_opt_ref_free(s);
        return -1;
    }
    memcpy(s->U, U, sizeof(double) * (size_t)L * k);
    memcpy(s->V, V, sizeof(double) * (size_t)K * k);
    memcpy(s->sigma, sigma, sizeof(double) * k);
    s->total_variance = 0.0;
    for (int i = 0; i < k; i++)
    {
        s->eigenvalues[i] = sigma[i] * sigma[i];
        s->total_variance += s->eigenvalues[i];
    }
    s->n_components = k;
    s->decomposed = true;
    return 0;
}

REFDRV_API int refdrv_reconstruct(const double *x, int N, int L, int k, const double *U,
                                  const double *V, const double *sigma, const int *group,
                                  int n_group, double *out)
{
    SSA_Opt_Ref s;
    if (refdrv_ctx_with(&s, x, N, L, k, U, V, sigma) != 0)
        return -1;
    int r = ssa_opt_ref_reconstruct(&s, group, n_group, out);
    ssa_opt_ref_free(&s);
    return r;
}

REFDRV_API int refdrv_wcorr(const double *x, int N, int L, int k, const double *U,
                            const double *V, const double *sigma, double *W)
{
    SSA_Opt_Ref s;
    if (refdrv_ctx_with(&s, x, N, L, k, U, V, sigma) != 0)
        return -1;
    int r = ssa_opt_ref_wcorr_matrix(&s, W);
    ssa_opt_ref_free(&s);
    return r;
}

REFDRV_API int refdrv_lrf(const double *x, int N, int L, int k, const double *U,
                          const double *V, const double *sigma, const int *group, int n_group,
                          double *R, double *verticality)
{
    SSA_Opt_Ref s;
    if (refdrv_ctx_with(&s, x, N, L, k, U, V, sigma) != 0)
        return -1;
    int r = ssa_opt_ref_compute_lrf(&s, group, n_group, R, verticality);
    ssa_opt_ref_free(&s);
    return r;
}

/* output has N + n_forecast entries (ssa_opt_ref.h:1660-1701). */
REFDRV_API int refdrv_forecast(const double *x, int N, int L, int k, const double *U,
                               const double *V, const double *sigma, const int *group,
                               int n_group, int n_forecast, double *out)
{
    SSA_Opt_Ref s;
    if (refdrv_ctx_with(&s, x, N, L, k, U, V, sigma) != 0)
        return -1;
    int r = ssa_opt_ref_forecast(&s, group, n_group, n_forecast, out);
    ssa_opt_ref_free(&s);
    return r;
}

/* The reference CPU path for one series: init, randomized decomposition (rng state `state`),
 * reconstruction of every component group in `groups` (n_groups groups of sizes
 * group_sizes[], concatenated) into recon (n_groups x N), and the k x k W-correlation.
 * Returns the number of components or -1. */
REFDRV_API int refdrv_pipeline(const double *x, int N, int L, int k, int p, uint64_t state,
                               const int *groups, const int *group_sizes, int n_groups,
                               double *sigma, double *recon, double *W)
{
    SSA_Opt_Ref s;
    memset(&s, 0, sizeof(s));
    if (ssa_opt_ref_init(&s, x, N, L) != 0)
        return -1;
    s.rng_state = state;
    if (ssa_opt_ref_decompose_randomized(&s, k, p) != 0)
    {
        ssa_opt_ref_free(&s);
        return -1;
    }
    int kk = s.n_components;
    memcpy(sigma, s.sigma, sizeof(double) * kk);
    int off = 0;
    for (int g = 0; g < n_groups; g++)
    {
        if (ssa_opt_ref_reconstruct(&s, groups + off, group_sizes[g], recon + (size_t)g * N) != 0)
        {
            ssa_opt_ref_free(&s);
            return -1;
        }
        off += group_sizes[g];
    }
    if (W && ssa_opt_ref_wcorr_matrix(&s, W) != 0)
    {
        ssa_opt_ref_free(&s);
        return -1;
    }
    ssa_opt_ref_free(&s);
    return kk;
}
