/* Checker driver around the reference's own MKL/ssa_opt.h (TEST INFRASTRUCTURE ONLY).
 *
 * This file compiles the unmodified reference header with SSA_OPT_IMPLEMENTATION against the
 * MKL-compatibility shim in oracle/mklshim/ (own DFTI FFT, VML loops, VSL draws from a
 * host-registered buffer, CBLAS/LAPACKE from scipy's OpenBLAS) and exports flat-array entry
 * points (prefix mkr_) for tests/ and for bench.py's CPU-baseline leg. Nothing in the product
 * (libssa.so) links it. Built by oracle/Makefile into oracle/_ref/libssa_mklshim.so.
 *
 * Every entry point runs a whole reference call sequence on a fresh context (init -> prepare ->
 * decompose -> ...), exactly as the reference's Python wrapper drives it
 * (MKL/py/ssa_wrapper.py:630-851), and copies the results out. Returns are the reference's
 * (0 / -1), or a component / iteration count where stated. */
#define SSA_OPT_IMPLEMENTATION
#include "ssa_opt.h"

#define MKR_EXPORT __attribute__((visibility("default")))

static void mkr_copy_factors(const SSA_Opt *s, double *sigma, double *U, double *V)
{
    const int k = s->n_components;
    if (sigma)
        memcpy(sigma, s->sigma, sizeof(double) * (size_t)k);
    if (U)
        memcpy(U, s->U, sizeof(double) * (size_t)k * (size_t)s->L);
    if (V)
        memcpy(V, s->V, sizeof(double) * (size_t)k * (size_t)s->K);
}

/* Randomized decomposition (MKL/ssa_opt.h:1685-1763): init, prepare(k, p),
 * decompose_randomized(k, p). Outputs sigma[k'], U[L x k'], V[K x k'] column-major,
 * total_variance; returns k' (components computed) or -1. */
MKR_EXPORT int mkr_randomized(const double *x, int N, int L, int k, int p, double *sigma,
                              double *U, double *V, double *total_var)
{
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0)
        return -1;
    int rc = -1;
    if (ssa_opt_prepare(&s, k, p) == 0 && ssa_opt_decompose_randomized(&s, k, p) == 0) {
        mkr_copy_factors(&s, sigma, U, V);
        if (total_var)
            *total_var = s.total_variance;
        rc = s.n_components;
    }
    ssa_opt_free(&s);
    return rc;
}

/* Block power decomposition (MKL/ssa_opt.h:1765-1933); uniform start blocks from the stream. */
MKR_EXPORT int mkr_block(const double *x, int N, int L, int k, int block, int max_iter,
                         double *sigma, double *U, double *V)
{
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0)
        return -1;
    int rc = -1;
    if (ssa_opt_decompose_block(&s, k, block, max_iter) == 0) {
        mkr_copy_factors(&s, sigma, U, V);
        rc = s.n_components;
    }
    ssa_opt_free(&s);
    return rc;
}

/* Sequential power decomposition (MKL/ssa_opt.h:1560-1678). */
MKR_EXPORT int mkr_sequential(const double *x, int N, int L, int k, int max_iter, double *sigma,
                              double *U, double *V)
{
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0)
        return -1;
    int rc = -1;
    if (ssa_opt_decompose(&s, k, max_iter) == 0) {
        mkr_copy_factors(&s, sigma, U, V);
        rc = s.n_components;
    }
    ssa_opt_free(&s);
    return rc;
}

/* Hankel matvec / adjoint through the reference's FFT path (MKL/ssa_opt.h:871-903). */
MKR_EXPORT int mkr_matvec(const double *x, int N, int L, const double *v, double *y, int adjoint)
{
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0)
        return -1;
    if (adjoint)
        ssa_opt_hankel_matvec_T(&s, v, y);
    else
        ssa_opt_hankel_matvec(&s, v, y);
    ssa_opt_free(&s);
    return 0;
}

/* The reference's decompose -> reconstruct -> W-correlation -> forecast sequence as the
 * Python wrapper runs it (randomized decomposition with oversampling p, uncached
 * reconstructions, ssa_opt_wcorr_matrix, ssa_opt_forecast). Any output pointer may be NULL to
 * skip that step. groups: concatenated indices, sizes[n_groups]; recon: n_groups x N.
 * w_mode: 0 none, 1 ssa_opt_wcorr_matrix without cached spectra, 2 ssa_opt_cache_ffts then
 * ssa_opt_wcorr_matrix_fast. fgroup/nf/h: forecast group and horizon (fc[h]); lrf_R[L-1] and
 * verticality from ssa_opt_compute_lrf of the same group. Returns k' or -1. */
MKR_EXPORT int mkr_pipeline(const double *x, int N, int L, int k, int p, const int *groups,
                            const int *sizes, int n_groups, double *recon, int w_mode, double *W,
                            const int *fgroup, int nf, int h, double *fc, double *lrf_R,
                            double *verticality, double *sigma)
{
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0)
        return -1;
    int rc = -1;
    if (ssa_opt_prepare(&s, k, p) != 0 || ssa_opt_decompose_randomized(&s, k, p) != 0)
        goto done;
    if (sigma)
        memcpy(sigma, s.sigma, sizeof(double) * (size_t)s.n_components);
    if (recon && groups && sizes) {
        int off = 0;
        for (int g = 0; g < n_groups; g++) {
            if (ssa_opt_reconstruct(&s, groups + off, sizes[g], recon + (size_t)g * N) != 0)
                goto done;
            off += sizes[g];
        }
    }
    if (W && w_mode == 1) {
        if (ssa_opt_wcorr_matrix(&s, W) != 0)
            goto done;
    } else if (W && w_mode == 2) {
        if (ssa_opt_cache_ffts(&s) != 0 || ssa_opt_wcorr_matrix_fast(&s, W) != 0)
            goto done;
    }
    if (fgroup && nf > 0) {
        if (lrf_R || verticality) {
            SSA_LRF lrf;
            if (ssa_opt_compute_lrf(&s, fgroup, nf, &lrf) != 0)
                goto done;
            if (lrf_R)
                memcpy(lrf_R, lrf.R, sizeof(double) * (size_t)(L - 1));
            if (verticality)
                *verticality = lrf.verticality;
            ssa_opt_lrf_free(&lrf);
        }
        if (fc && h > 0 && ssa_opt_forecast(&s, fgroup, nf, h, fc) != 0)
            goto done;
    }
    rc = s.n_components;
done:
    ssa_opt_free(&s);
    return rc;
}

/* W-correlation consumers on a randomized decomposition (MKL/ssa_opt.h:2551-2756):
 * pair_ij[n_pairs] = ssa_opt_wcorr_pair for the index pairs (pi[t], pj[t]); component stats
 * (gaps[k-1], cumulative_var[k], second_diff[k], suggested_signal); periodic pairs with the
 * given thresholds (pairs_out[2 * max_pairs], returns the count in *n_periodic). gaps are the
 * reference's ratios sigma_i / sigma_{i+1}; second_diff has k entries (zero at both ends). */
MKR_EXPORT int mkr_wcorr_consumers(const double *x, int N, int L, int k, int p, const int *pi,
                                   const int *pj, int n_pairs, double *pair_out, double *gaps,
                                   double *cumvar, double *second_diff, int *suggested,
                                   int *pairs_out, int max_pairs, double sv_tol,
                                   double wcorr_thresh, int *n_periodic)
{
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0)
        return -1;
    int rc = -1;
    if (ssa_opt_prepare(&s, k, p) != 0 || ssa_opt_decompose_randomized(&s, k, p) != 0)
        goto done;
    for (int t = 0; t < n_pairs; t++)
        pair_out[t] = ssa_opt_wcorr_pair(&s, pi[t], pj[t]);
    {
        SSA_ComponentStats st;
        if (ssa_opt_component_stats(&s, &st) != 0)
            goto done;
        const int n = st.n;
        if (gaps && n > 1)
            memcpy(gaps, st.gaps, sizeof(double) * (size_t)(n - 1));
        if (cumvar)
            memcpy(cumvar, st.cumulative_var, sizeof(double) * (size_t)n);
        if (second_diff)
            memcpy(second_diff, st.second_diff, sizeof(double) * (size_t)n);
        if (suggested)
            *suggested = st.suggested_signal;
        ssa_opt_component_stats_free(&st);
    }
    if (pairs_out && n_periodic)
        *n_periodic = ssa_opt_find_periodic_pairs(&s, pairs_out, max_pairs, sv_tol, wcorr_thresh);
    rc = s.n_components;
done:
    ssa_opt_free(&s);
    return rc;
}

/* Multichannel SSA (MKL/ssa_opt.h:3908-4283): X is M x N row-major (channel m at X[m N]).
 * Outputs sigma[k'], U[(M L) x k'], V[K x k'], recon[M x N] of `group` for every channel,
 * contributions[M x k'] (series_contributions). Returns k' or -1. */
MKR_EXPORT int mkr_mssa(const double *X, int M, int N, int L, int k, int p, double *sigma,
                        double *U, double *V, const int *group, int ng, double *recon,
                        double *contrib)
{
    MSSA_Opt m;
    if (mssa_opt_init(&m, X, M, N, L) != 0)
        return -1;
    int rc = -1;
    if (mssa_opt_decompose(&m, k, p) != 0)
        goto done;
    const int kk = m.n_components;
    if (sigma)
        memcpy(sigma, m.sigma, sizeof(double) * (size_t)kk);
    if (U)
        memcpy(U, m.U, sizeof(double) * (size_t)kk * (size_t)M * (size_t)L);
    if (V)
        memcpy(V, m.V, sizeof(double) * (size_t)kk * (size_t)m.K);
    if (recon && group && ng > 0 && mssa_opt_reconstruct_all(&m, group, ng, recon) != 0)
        goto done;
    if (contrib && mssa_opt_series_contributions(&m, contrib) != 0)
        goto done;
    rc = kk;
done:
    mssa_opt_free(&m);
    return rc;
}

/* Cadzow (MKL/ssa_opt.h:3165-3442). mode 0: ssa_opt_cadzow; 1: ssa_opt_cadzow_weighted(alpha);
 * 2: ssa_opt_cadzow_inplace on a context initialised with x (out = the context's final
 * reconstruction of components 0..rank-1 is not exposed by the reference, so out receives the
 * signal the context holds after the call: ssa_opt_reconstruct of 0..rank-1). Returns the
 * reference's return value (iterations or -1). */
MKR_EXPORT int mkr_cadzow(const double *x, int N, int L, int rank, int max_iter, double tol,
                          int mode, double alpha, double *out, int *iterations, double *final_diff,
                          double *converged)
{
    SSA_CadzowResult r;
    memset(&r, 0, sizeof(r));
    int rc;
    if (mode == 0) {
        rc = ssa_opt_cadzow(x, N, L, rank, max_iter, tol, out, &r);
    } else if (mode == 1) {
        rc = ssa_opt_cadzow_weighted(x, N, L, rank, max_iter, tol, alpha, out, &r);
    } else {
        SSA_Opt s;
        if (ssa_opt_init(&s, x, N, L) != 0)
            return -1;
        if (ssa_opt_prepare(&s, rank, 8) != 0) {
            ssa_opt_free(&s);
            return -1;
        }
        rc = ssa_opt_cadzow_inplace(&s, rank, max_iter, tol, &r);
        if (rc >= 0 && out) {
            int *g = malloc(sizeof(int) * (size_t)rank);
            for (int i = 0; i < rank; i++)
                g[i] = i;
            if (!s.decomposed || ssa_opt_reconstruct(&s, g, rank, out) != 0)
                rc = -1;
            free(g);
        }
        ssa_opt_free(&s);
    }
    if (iterations)
        *iterations = r.iterations;
    if (final_diff)
        *final_diff = r.final_diff;
    if (converged)
        *converged = r.converged;
    return rc;
}

/* Gap filling (MKL/ssa_opt.h:3498-3878): x is modified in place (NaN = gap). simple != 0 runs
 * ssa_opt_gapfill_simple. Returns the reference's return value. */
MKR_EXPORT int mkr_gapfill(double *x, int N, int L, int rank, int max_iter, double tol, int simple,
                           int *iterations, double *final_diff, int *converged, int *n_gaps)
{
    SSA_GapFillResult r;
    memset(&r, 0, sizeof(r));
    const int rc = simple ? ssa_opt_gapfill_simple(x, N, L, rank, &r)
                          : ssa_opt_gapfill(x, N, L, rank, max_iter, tol, &r);
    if (iterations)
        *iterations = r.iterations;
    if (final_diff)
        *final_diff = r.final_diff;
    if (converged)
        *converged = r.converged;
    if (n_gaps)
        *n_gaps = r.n_gaps;
    return rc;
}

/* ESPRIT (MKL/ssa_opt.h:4304-4558) on a randomized decomposition (k, p). Outputs per
 * component of the group: periods, frequencies, moduli, rates. Returns n or -1. */
MKR_EXPORT int mkr_parestimate(const double *x, int N, int L, int k, int p, const int *group,
                               int ng, double *periods, double *freqs, double *moduli,
                               double *rates)
{
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0)
        return -1;
    int rc = -1;
    if (ssa_opt_prepare(&s, k, p) != 0 || ssa_opt_decompose_randomized(&s, k, p) != 0)
        goto done;
    SSA_ParEstimate pe;
    memset(&pe, 0, sizeof(pe));
    if (ssa_opt_parestimate(&s, group, ng, &pe) != 0)
        goto done;
    const int n = pe.n_components;
    if (periods)
        memcpy(periods, pe.periods, sizeof(double) * (size_t)n);
    if (freqs)
        memcpy(freqs, pe.frequencies, sizeof(double) * (size_t)n);
    if (moduli)
        memcpy(moduli, pe.moduli, sizeof(double) * (size_t)n);
    if (rates)
        memcpy(rates, pe.rates, sizeof(double) * (size_t)n);
    ssa_opt_parestimate_free(&pe);
    rc = n;
done:
    ssa_opt_free(&s);
    return rc;
}

/* An R-forecast request on a resident series, timed: the decomposition (init, prepare,
 * decompose_randomized) is made first and not timed, then ssa_opt_forecast(fgroup, h) is timed
 * with the monotonic clock (MKL/ssa_opt.h:2843-2867: reconstruct the group, LRF, recurrence).
 * *seconds receives the forecast's time. Returns 0 or -1. */
#include <time.h>
MKR_EXPORT int mkr_forecast_resident(const double *x, int N, int L, int k, int p, const int *fgroup,
                                     int nf, int h, double *fc, double *seconds)
{
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0)
        return -1;
    int rc = -1;
    if (ssa_opt_prepare(&s, k, p) == 0 && ssa_opt_decompose_randomized(&s, k, p) == 0) {
        struct timespec t0, t1;
        clock_gettime(CLOCK_MONOTONIC, &t0);
        rc = ssa_opt_forecast(&s, fgroup, nf, h, fc);
        clock_gettime(CLOCK_MONOTONIC, &t1);
        if (seconds)
            *seconds = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
    }
    ssa_opt_free(&s);
    return rc;
}

/* FFT length and batch size the reference picks for (N, L) (MKL/ssa_opt.h:1047-1092). */
MKR_EXPORT int mkr_dims(const double *x, int N, int L, int *fft_len, int *batch_size)
{
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0)
        return -1;
    if (fft_len)
        *fft_len = s.fft_len;
    if (batch_size)
        *batch_size = s.batch_size;
    ssa_opt_free(&s);
    return 0;
}
