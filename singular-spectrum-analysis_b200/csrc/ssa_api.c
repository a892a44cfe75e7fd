/*
 * The SSA-Opt C API (MKL/ssa_opt.h:318-430) on the B200 device engine, one series per context.
 *
 * Every call validates its arguments exactly where the reference does, enqueues the device
 * pipeline on the context's stream, waits for it and mirrors results into the host fields of
 * SSA_Opt (sigma, eigenvalues, U, V). Return codes follow the reference: 0 / -1, counts for
 * the getters, 0.0 from double-valued getters on error.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "ssa_engine.h"
#include "../../include/ssa_opt.h"

struct ssa_gpu_ctx
{
    ssa_engine e;
    int engine_ok;
    int kp_cap, k_cap;          /* prepared capacity */
    int spectra_valid;          /* device spectra of sigma_i u_i and v_i are current */
    int wcorr_valid;            /* e.W holds the W-correlation of the current decomposition */
    int *d_group;
    int group_cap;
    double *d_out;              /* N (+ forecast) doubles */
    double *d_lrf;              /* R (L) + buf (L + h) + out (h) + verticality */
    size_t lrf_cap;
    int *d_status;
    float *h_stage;             /* pinned float staging, max(L, K) * k_cap */
    size_t stage_cap;
    float *d_omega;             /* K x kp caller-supplied test matrix (float) */
};

#define SSA_DEFAULT_SEED 42ULL

static int imin(int a, int b) { return a < b ? a : b; }

static void gpu_free(struct ssa_gpu_ctx *g)
{
    if (!g)
        return;
    if (g->engine_ok)
    {
        /* the context's buffers come from the engine's allocator (recycled or plain) */
        cudaStreamSynchronize(g->e.st);
        ssae_dfree(&g->e, g->d_group);
        ssae_dfree(&g->e, g->d_out);
        ssae_dfree(&g->e, g->d_lrf);
        ssae_dfree(&g->e, g->d_status);
        ssae_dfree(&g->e, g->d_omega);
        ssae_pinned_free(&g->e, g->h_stage, g->stage_cap * sizeof(float));
        ssae_destroy(&g->e);
    }
    free(g);
}

static int sync_ok(struct ssa_gpu_ctx *g)
{
    if (cudaStreamSynchronize(g->e.st) != cudaSuccess)
        return -1;
    return 0;
}

static int ensure_group(struct ssa_gpu_ctx *g, const int *group, int n)
{
    if (n > g->group_cap)
    {
        ssae_dfree(&g->e, g->d_group);
        g->d_group = NULL;
        int cap = n < 64 ? 64 : n;
        if (ssae_dalloc(&g->e, (void **)&g->d_group, sizeof(int) * cap) != 0)
        {
            g->group_cap = 0;
            return -1;
        }
        g->group_cap = cap;
    }
    return cudaMemcpyAsync(g->d_group, group, sizeof(int) * n, cudaMemcpyHostToDevice, g->e.st) == cudaSuccess ? 0 : -1;
}

static int ensure_stage(struct ssa_gpu_ctx *g, size_t floats)
{
    if (floats <= g->stage_cap)
        return 0;
    if (g->h_stage)
    {
        if (cudaStreamSynchronize(g->e.st) != cudaSuccess)
            return -1;
        ssae_pinned_free(&g->e, g->h_stage, g->stage_cap * sizeof(float));
    }
    g->h_stage = NULL;
    g->stage_cap = 0;
    size_t cap = 0;
    if (ssae_pinned(&g->e, floats * sizeof(float), (void **)&g->h_stage, &cap) != 0)
    {
        g->h_stage = NULL;
        return -1;
    }
    g->stage_cap = cap / sizeof(float);
    return 0;
}

/* Copy the signal spectrum into the host field fft_x (interleaved, r2c_len complex). */
static int mirror_spectrum(SSA_Opt *ssa)
{
    struct ssa_gpu_ctx *g = ssa->gpu;
    const int n = 2 * ssa->r2c_len;
    if (ensure_stage(g, (size_t)n) != 0)
        return -1;
    if (cudaMemcpyAsync(g->h_stage, g->e.X, sizeof(float) * n, cudaMemcpyDeviceToHost, g->e.st) != cudaSuccess)
        return -1;
    if (sync_ok(g) != 0)
        return -1;
    for (int i = 0; i < n; i++)
        ssa->fft_x[i] = (double)g->h_stage[i];
    return 0;
}

int ssa_opt_init(SSA_Opt *ssa, const ssa_real *x, int N, int L)
{
    if (!ssa || !x || N < 4 || L < 2 || L > N - 1)
        return -1;
    memset(ssa, 0, sizeof(SSA_Opt));
    const int logh = ssad_logh_for(N);
    if (logh > SSA_MAX_LOGH_ALL)
        return -1;
    ssa->N = N;
    ssa->L = L;
    ssa->K = N - L + 1;
    ssa->fft_len = 2 << logh;
    ssa->r2c_len = (1 << logh) + 1;
    ssa->batch_size = 1;
    struct ssa_gpu_ctx *g = (struct ssa_gpu_ctx *)calloc(1, sizeof(*g));
    if (!g)
        return -1;
    ssa->gpu = g;
    /* Engine with room for k + p = min(SSA_MAX_KP, L, K) columns; prepare() narrows it. */
    int kp = imin(SSA_MAX_KP, imin(L, ssa->K));
    if (ssae_create(&g->e, 1, N, L, kp, kp, NULL) != 0)
    {
        free(g);
        ssa->gpu = NULL;
        return -1;
    }
    g->engine_ok = 1;
    ssa->fft_x = (double *)malloc(sizeof(double) * 2 * ssa->r2c_len);
    ssa->ws_real = (double *)malloc(sizeof(double) * (N > ssa->fft_len ? N : ssa->fft_len));
    ssa->ws_complex = (double *)malloc(sizeof(double) * 2 * ssa->r2c_len);
    ssa->inv_diag_count = (double *)malloc(sizeof(double) * N);
    if (!ssa->fft_x || !ssa->ws_real || !ssa->ws_complex || !ssa->inv_diag_count ||
        ssae_dalloc(&g->e, (void **)&g->d_out, sizeof(double) * (size_t)N) != 0)
    {
        ssa_opt_free(ssa);
        return -1;
    }
    for (int t = 0; t < N; t++)
    {
        int c = imin(imin(t + 1, L), imin(ssa->K, N - t));
        ssa->inv_diag_count[t] = c > 0 ? 1.0 / c : 0.0;
    }
    if (cudaMemcpyAsync(g->e.x64, x, sizeof(double) * N, cudaMemcpyHostToDevice, g->e.st) != cudaSuccess ||
        ssae_signal_spectrum(&g->e, g->e.x64, 1) != 0 || mirror_spectrum(ssa) != 0)
    {
        ssa_opt_free(ssa);
        return -1;
    }
    ssae_reset_jobs(&g->e);
    ssa->initialized = true;
    return 0;
}

static void free_results(SSA_Opt *ssa)
{
    free(ssa->U);
    free(ssa->V);
    free(ssa->sigma);
    free(ssa->eigenvalues);
    ssa->U = ssa->V = ssa->sigma = ssa->eigenvalues = NULL;
}

void ssa_opt_free(SSA_Opt *ssa)
{
    if (!ssa)
        return;
    gpu_free(ssa->gpu);
    free_results(ssa);
    free(ssa->fft_x);
    free(ssa->ws_real);
    free(ssa->ws_complex);
    free(ssa->inv_diag_count);
    free(ssa->decomp_Omega);
    memset(ssa, 0, sizeof(SSA_Opt));
}

void ssa_opt_free_prepared(SSA_Opt *ssa)
{
    if (!ssa)
        return;
    free(ssa->decomp_Omega);
    ssa->decomp_Omega = NULL;
    ssa->prepared_kp = 0;
    ssa->prepared_lwork = 0;
    ssa->prepared = false;
}

static int alloc_results(SSA_Opt *ssa, int k)
{
    free_results(ssa);
    ssa->U = (double *)calloc((size_t)ssa->L * k, sizeof(double));
    ssa->V = (double *)calloc((size_t)ssa->K * k, sizeof(double));
    ssa->sigma = (double *)calloc((size_t)k, sizeof(double));
    ssa->eigenvalues = (double *)calloc((size_t)k, sizeof(double));
    if (!ssa->U || !ssa->V || !ssa->sigma || !ssa->eigenvalues)
    {
        free_results(ssa);
        return -1;
    }
    return 0;
}

int ssa_opt_prepare(SSA_Opt *ssa, int max_k, int oversampling)
{
    if (!ssa || !ssa->initialized || max_k < 1)
        return -1;
    ssa_opt_free_prepared(ssa);
    const int L = ssa->L, K = ssa->K;
    const int p = oversampling <= 0 ? 8 : oversampling;
    int kp = max_k + p;
    kp = imin(kp, imin(L, K));
    const int actual_k = imin(max_k, kp);
    if (kp > SSA_MAX_KP)
        return -1;
    ssa->decomp_Omega = (double *)malloc(sizeof(double) * (size_t)K * kp);
    if (!ssa->decomp_Omega || alloc_results(ssa, actual_k) != 0)
    {
        ssa_opt_free_prepared(ssa);
        return -1;
    }
    ssa->n_components = actual_k;
    ssa->prepared_kp = kp;
    ssa->prepared = true;
    return 0;
}

int ssa_opt_update_signal(SSA_Opt *ssa, const ssa_real *new_x)
{
    if (!ssa || !ssa->initialized || !new_x)
        return -1;
    struct ssa_gpu_ctx *g = ssa->gpu;
    ssa_opt_free_cached_ffts(ssa);
    ssa->decomposed = false;
    g->spectra_valid = 0;
    g->wcorr_valid = 0;
    ssae_reset_jobs(&g->e);
    if (cudaMemcpyAsync(g->e.x64, new_x, sizeof(double) * ssa->N, cudaMemcpyHostToDevice, g->e.st) != cudaSuccess ||
        ssae_signal_spectrum(&g->e, g->e.x64, 1) != 0 || mirror_spectrum(ssa) != 0)
        return -1;
    return 0;
}

/* Download U (L x k), V (K x k), sigma into the host fields. */
static int mirror_results(SSA_Opt *ssa, int k)
{
    struct ssa_gpu_ctx *g = ssa->gpu;
    ssa_engine *e = &g->e;
    const int L = ssa->L, K = ssa->K;
    if (ensure_stage(g, (size_t)(L > K ? L : K) * k) != 0)
        return -1;
    if (cudaMemcpy2DAsync(g->h_stage, sizeof(float) * L, e->Y, sizeof(float) * e->ldL, sizeof(float) * L, k,
                          cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
        cudaMemcpyAsync(ssa->sigma, e->sigma, sizeof(double) * k, cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
        sync_ok(g) != 0)
        return -1;
    for (size_t i = 0; i < (size_t)L * k; i++)
        ssa->U[i] = (double)g->h_stage[i];
    if (cudaMemcpy2DAsync(g->h_stage, sizeof(float) * K, e->Z, sizeof(float) * e->ldK, sizeof(float) * K, k,
                          cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
        sync_ok(g) != 0)
        return -1;
    for (size_t i = 0; i < (size_t)K * k; i++)
        ssa->V[i] = (double)g->h_stage[i];
    ssa->total_variance = 0.0;
    for (int i = 0; i < k; i++)
    {
        ssa->eigenvalues[i] = ssa->sigma[i] * ssa->sigma[i];
        ssa->total_variance += ssa->eigenvalues[i];
    }
    return 0;
}

static int check_status(struct ssa_gpu_ctx *g)
{
    int st = 0;
    if (cudaMemcpy(&st, g->e.status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    return st == 0 ? 0 : -1;
}

/* Shared body of the randomized decompositions: Omega = host matrix (K x kp, column-major,
 * double) or NULL for the device generator. */
static int decompose_randomized_impl(SSA_Opt *ssa, int k, int oversampling, int q, const double *Omega)
{
    if (!ssa || !ssa->initialized || k < 1 || q < 0)
        return -1;
    ssa_opt_free_cached_ffts(ssa);
    const int L = ssa->L, K = ssa->K;
    const int p = oversampling <= 0 ? 8 : oversampling;
    int kp = imin(k + p, imin(L, K));
    k = imin(k, kp);
    if (!ssa->prepared || kp > ssa->prepared_kp)
        return -1;
    struct ssa_gpu_ctx *g = ssa->gpu;
    ssa_engine *e = &g->e;
    ssae_reset_jobs(e);
    g->spectra_valid = 0;
    g->wcorr_valid = 0;
    ssa->decomposed = false;
    ssa->n_components = k;
    int rc = 0;
    if (Omega)
    {
        if (ensure_stage(g, (size_t)K * kp) != 0)
            return -1;
        for (size_t i = 0; i < (size_t)K * kp; i++)
            g->h_stage[i] = (float)Omega[i];
        rc |= cudaMemcpy2DAsync(e->Z, sizeof(float) * e->ldK, g->h_stage, sizeof(float) * K, sizeof(float) * K, kp,
                                cudaMemcpyHostToDevice, e->st) != cudaSuccess;
        rc |= ssae_decompose(e, 1, kp, k, q, e->Z, e->ldK, 0) != 0;
    }
    else
    {
        const unsigned long long seed = SSA_DEFAULT_SEED + 0x100000000ULL * (unsigned long long)ssa->rng_calls;
        ssa->rng_calls++;
        rc |= ssae_decompose(e, 1, kp, k, q, NULL, 0, seed) != 0;
    }
    if (rc || sync_ok(g) != 0 || check_status(g) != 0 || mirror_results(ssa, k) != 0)
        return -1;
    ssa->decomposed = true;
    return 0;
}

int ssa_opt_decompose_randomized(SSA_Opt *ssa, int k, int oversampling)
{
    return decompose_randomized_impl(ssa, k, oversampling, 0, NULL);
}

int ssa_opt_decompose_randomized_ex(SSA_Opt *ssa, int k, int oversampling, int power_iters, const double *Omega)
{
    return decompose_randomized_impl(ssa, k, oversampling, power_iters, Omega);
}

/* Block power iteration with Rayleigh-Ritz (MKL/ssa_opt.h:1765-1933) on the device. V0: host
 * K x k column-major start blocks (block i = its columns), or NULL for the library generator.
 * Like the reference it (re)allocates the result arrays on every call. */
static int decompose_block_impl(SSA_Opt *ssa, int k, int block_size, int max_iter, const double *V0)
{
    if (!ssa || !ssa->initialized || k < 1 || block_size < 1)
        return -1;
    ssa_opt_free_cached_ffts(ssa);
    const int L = ssa->L, K = ssa->K;
    const int b = imin(block_size, imin(k, imin(L, K)));
    k = imin(k, imin(L, K));
    if (k > SSA_MAX_KP || max_iter < 0)
        return -1;
    (void)b;
    struct ssa_gpu_ctx *g = ssa->gpu;
    ssa_engine *e = &g->e;
    ssae_reset_jobs(e);
    g->spectra_valid = 0;
    g->wcorr_valid = 0;
    ssa->decomposed = false;
    if (alloc_results(ssa, k) != 0)
        return -1;
    ssa->n_components = k;
    const float *d_V0 = NULL;
    if (V0)
    {
        if (ssae_ensure_block(e, imin(block_size, k)) != 0 || ensure_stage(g, (size_t)K * k) != 0)
            return -1;
        for (size_t i = 0; i < (size_t)K * k; i++)
            g->h_stage[i] = (float)V0[i];
        /* staged in the permutation buffer Vt, which the decomposition only uses at its end */
        if (cudaMemcpyAsync(e->Vt, g->h_stage, sizeof(float) * (size_t)K * k, cudaMemcpyHostToDevice, e->st) !=
            cudaSuccess)
            return -1;
        d_V0 = e->Vt;
    }
    const unsigned long long seed =
        (SSA_DEFAULT_SEED + 0x100000000ULL * (unsigned long long)ssa->rng_calls) ^ 0xB10CB10CB10CB10CULL;
    ssa->rng_calls++;
    if (ssae_decompose_block(e, 1, k, block_size, max_iter, d_V0, K, seed) != 0 || sync_ok(g) != 0 ||
        check_status(g) != 0 || mirror_results(ssa, k) != 0)
        return -1;
    ssa->decomposed = true;
    return 0;
}

int ssa_opt_decompose_block(SSA_Opt *ssa, int k, int block_size, int max_iter)
{
    return decompose_block_impl(ssa, k, block_size, max_iter, NULL);
}

int ssa_opt_decompose_block_ex(SSA_Opt *ssa, int k, int block_size, int max_iter, const double *V0)
{
    return decompose_block_impl(ssa, k, block_size, max_iter, V0);
}

/* Sequential power iteration (MKL/ssa_opt.h:1560-1678) computes one component at a time with
 * deflation against the earlier ones; on the device it runs as block power iteration with
 * blocks of one column, which has the same fixed points (the reference's early stop on
 * convergence is not reproduced: all max_iter iterations run). */
int ssa_opt_decompose(SSA_Opt *ssa, int k, int max_iter)
{
    if (!ssa || !ssa->initialized || k < 1)
        return -1;
    return decompose_block_impl(ssa, k, 1, max_iter, NULL);
}

/* ssa_opt_extend (MKL/ssa_opt.h:1935-2056) is outside the accelerated path: it reports failure. */
int ssa_opt_extend(SSA_Opt *ssa, int additional_k, int max_iter)
{
    if (!ssa || !ssa->decomposed || additional_k < 1 || max_iter < 0)
        return -1;
    ssa_opt_free_cached_ffts(ssa);
    const int L = ssa->L, K = ssa->K, old_k = ssa->n_components;
    const int new_k = imin(old_k + additional_k, imin(L, K));
    if (new_k <= old_k)
        return 0;
    struct ssa_gpu_ctx *g = ssa->gpu;
    ssa_engine *e = &g->e;
    if (new_k > e->k || new_k > SSA_MAX_KP)
        return -1;
    ssae_reset_jobs(e);
    g->spectra_valid = 0;
    g->wcorr_valid = 0;
    const unsigned long long seed =
        (SSA_DEFAULT_SEED + 0x100000000ULL * (unsigned long long)ssa->rng_calls) ^ 0xB10CB10CB10CB10CULL;
    ssa->rng_calls++;
    ssa->decomposed = false;
    if (ssae_extend(e, old_k, new_k, max_iter, seed) != 0 || sync_ok(g) != 0 || check_status(g) != 0 ||
        alloc_results(ssa, new_k) != 0 || mirror_results(ssa, new_k) != 0)
        return -1;
    ssa->n_components = new_k;
    ssa->decomposed = true;
    return 0;
}

/* ---- spectra cache and reconstruction -------------------------------------------------- */

static int ensure_spectra(const SSA_Opt *ssa)
{
    struct ssa_gpu_ctx *g = ssa->gpu;
    if (g->spectra_valid)
        return 0;
    if (ssae_spectra(&g->e, 1, ssa->n_components) != 0)
        return -1;
    g->spectra_valid = 1;
    return 0;
}

int ssa_opt_cache_ffts(SSA_Opt *ssa)
{
    if (!ssa || !ssa->decomposed)
        return -1;
    ssae_reset_jobs(&ssa->gpu->e);
    if (ensure_spectra(ssa) != 0 || sync_ok(ssa->gpu) != 0)
        return -1;
    ssa->fft_cached = true;
    return 0;
}

void ssa_opt_free_cached_ffts(SSA_Opt *ssa)
{
    if (!ssa)
        return;
    ssa->fft_cached = false;
    /* Device spectra stay allocated and are recomputed after the next decomposition. */
}

/* Device reconstruction of `group` into g->d_out (not synchronised). */
static int recon_device(const SSA_Opt *ssa, const int *group, int n_group)
{
    struct ssa_gpu_ctx *g = ssa->gpu;
    if (ensure_spectra(ssa) != 0 || ensure_group(g, group, n_group) != 0)
        return -1;
    return ssae_recon_group(&g->e, 0, ssa->n_components, g->d_group, n_group, g->d_out) != 0 ? -1 : 0;
}

int ssa_opt_reconstruct(const SSA_Opt *ssa, const int *group, int n_group, ssa_real *output)
{
    if (!ssa || !ssa->decomposed || !group || !output || n_group < 1)
        return -1;
    struct ssa_gpu_ctx *g = ssa->gpu;
    ssae_reset_jobs(&g->e);
    if (recon_device(ssa, group, n_group) != 0 ||
        cudaMemcpyAsync(output, g->d_out, sizeof(double) * ssa->N, cudaMemcpyDeviceToHost, g->e.st) != cudaSuccess ||
        sync_ok(g) != 0)
        return -1;
    return 0;
}

/* ---- W-correlation ---------------------------------------------------------------------- */

static int wcorr_device(const SSA_Opt *ssa)
{
    struct ssa_gpu_ctx *g = ssa->gpu;
    if (g->wcorr_valid)
        return 0;
    const int k = ssa->n_components;
    ssae_reset_jobs(&g->e);
    if (ssae_elem_recon(&g->e, 1, k) != 0 || ssae_wcorr(&g->e, 1, k) != 0 || sync_ok(g) != 0)
        return -1;
    g->wcorr_valid = 1;
    return 0;
}

int ssa_opt_wcorr_matrix(const SSA_Opt *ssa, ssa_real *W)
{
    if (!ssa || !ssa->decomposed || !W)
        return -1;
    struct ssa_gpu_ctx *g = ssa->gpu;
    const int k = ssa->n_components;
    if (wcorr_device(ssa) != 0 ||
        cudaMemcpy(W, g->e.W, sizeof(double) * k * k, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    return 0;
}

int ssa_opt_wcorr_matrix_fast(const SSA_Opt *ssa, ssa_real *W) { return ssa_opt_wcorr_matrix(ssa, W); }

ssa_real ssa_opt_wcorr_pair(const SSA_Opt *ssa, int i, int j)
{
    if (!ssa || !ssa->decomposed || i < 0 || i >= ssa->n_components || j < 0 || j >= ssa->n_components)
        return 0.0;
    struct ssa_gpu_ctx *g = ssa->gpu;
    const int k = ssa->n_components;
    double w = 0.0;
    if (wcorr_device(ssa) != 0 ||
        cudaMemcpy(&w, g->e.W + (size_t)i * k + j, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return 0.0;
    return w;
}

/* ---- LRF / forecast --------------------------------------------------------------------- */

static int ensure_lrf(struct ssa_gpu_ctx *g, size_t doubles)
{
    if (doubles <= g->lrf_cap)
        return 0;
    ssae_dfree(&g->e, g->d_lrf);
    g->d_lrf = NULL;
    g->lrf_cap = 0;
    if (ssae_dalloc(&g->e, (void **)&g->d_lrf, sizeof(double) * doubles) != 0)
        return -1;
    if (!g->d_status && ssae_dalloc(&g->e, (void **)&g->d_status, sizeof(int)) != 0)
        return -1;
    g->lrf_cap = doubles;
    return 0;
}

/* LRF of `group` and, with h > 0, the forecast over the reconstruction of the group.
 * Host outputs: R (L-1, may be NULL), verticality, fc (h). Returns 0 or -1 (verticality). */
/* LRF of the group and h steps of the recurrence on the device (k_lrf). The recurrence starts
 * from the last L-1 values of the group's reconstruction, or of `base_tail` (L-1 host values)
 * when that is given (no reconstruction then). */
static int lrf_forecast_from(const SSA_Opt *ssa, const int *group, int n_group, int h, double *R, double *vert,
                             double *fc, double *recon_out, const double *base_tail)
{
    struct ssa_gpu_ctx *g = ssa->gpu;
    const int L = ssa->L, N = ssa->N;
    if (n_group > SSA_MAX_KP)
        return -1;
    ssae_reset_jobs(&g->e);
    if (ensure_lrf(g, (size_t)(L - 1) + (size_t)(L - 1 + h) + (size_t)h + 1) != 0)
        return -1;
    double *dR = g->d_lrf, *dbuf = dR + (L - 1), *dout = dbuf + (L - 1 + h), *dvert = dout + h;
    if (base_tail)
    {
        /* the caller's window goes where the reconstruction would be (L - 1 <= N doubles) */
        if (ensure_group(g, group, n_group) != 0 ||
            cudaMemcpyAsync(g->d_out, base_tail, sizeof(double) * (size_t)(L - 1), cudaMemcpyHostToDevice,
                            g->e.st) != cudaSuccess)
            return -1;
    }
    else if (recon_device(ssa, group, n_group) != 0)
        return -1;
    ssa_lrf_job J;
    memset(&J, 0, sizeof(J));
    J.U = g->e.Y;
    J.group = g->d_group;
    J.recon = g->d_out;
    J.R = dR;
    J.buf = dbuf;
    J.out = dout;
    J.verticality = dvert;
    J.status = g->d_status;
    J.ld = g->e.ldL;
    J.L = L;
    J.N = base_tail ? L - 1 : N;
    J.n_group = n_group;
    J.h = h;
    J.k = ssa->n_components;
    void *d = ssae_push_jobs(&g->e, &J, sizeof(J));
    if (!d || cudaMemsetAsync(g->d_status, 0, sizeof(int), g->e.st) != cudaSuccess ||
        ssad_lrf((const ssa_lrf_job *)d, 1, g->e.st) != 0)
        return -1;
    int st = 0;
    if (cudaMemcpyAsync(&st, g->d_status, sizeof(int), cudaMemcpyDeviceToHost, g->e.st) != cudaSuccess ||
        cudaMemcpyAsync(vert, dvert, sizeof(double), cudaMemcpyDeviceToHost, g->e.st) != cudaSuccess ||
        sync_ok(g) != 0)
        return -1;
    if (st != 0)
        return -1;
    if (R && cudaMemcpy(R, dR, sizeof(double) * (L - 1), cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    if (h > 0 && cudaMemcpy(fc, dout, sizeof(double) * h, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    if (recon_out && cudaMemcpy(recon_out, g->d_out, sizeof(double) * N, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    return 0;
}

static int lrf_forecast(const SSA_Opt *ssa, const int *group, int n_group, int h, double *R, double *vert,
                        double *fc, double *recon_out)
{
    return lrf_forecast_from(ssa, group, n_group, h, R, vert, fc, recon_out, NULL);
}

static int group_in_range(const SSA_Opt *ssa, const int *group, int n_group)
{
    for (int i = 0; i < n_group; i++)
        if (group[i] < 0 || group[i] >= ssa->n_components)
            return 0;
    return 1;
}

int ssa_opt_compute_lrf(const SSA_Opt *ssa, const int *group, int n_group, SSA_LRF *lrf)
{
    if (!ssa || !ssa->decomposed || !group || !lrf || n_group < 1)
        return -1;
    memset(lrf, 0, sizeof(SSA_LRF));
    lrf->L = ssa->L;
    lrf->valid = false;
    if (!group_in_range(ssa, group, n_group))
        return -1;
    lrf->R = (double *)malloc(sizeof(double) * (ssa->L - 1));
    if (!lrf->R)
        return -1;
    double vert = 0.0;
    int rc = lrf_forecast(ssa, group, n_group, 0, lrf->R, &vert, NULL, NULL);
    lrf->verticality = vert;
    if (rc != 0)
    {
        free(lrf->R);
        lrf->R = NULL;
        return -1;
    }
    lrf->valid = true;
    return 0;
}

void ssa_opt_lrf_free(SSA_LRF *lrf)
{
    if (!lrf)
        return;
    free(lrf->R);
    memset(lrf, 0, sizeof(SSA_LRF));
}

int ssa_opt_forecast(const SSA_Opt *ssa, const int *group, int n_group, int n_forecast, ssa_real *output)
{
    if (!ssa || !ssa->decomposed || !group || !output || n_group < 1 || n_forecast < 1)
        return -1;
    if (!group_in_range(ssa, group, n_group))
        return -1;
    double vert;
    return lrf_forecast(ssa, group, n_group, n_forecast, NULL, &vert, output, NULL);
}

int ssa_opt_forecast_full(const SSA_Opt *ssa, const int *group, int n_group, int n_forecast, ssa_real *output)
{
    if (!ssa || !ssa->decomposed || !group || !output || n_group < 1 || n_forecast < 1)
        return -1;
    if (!group_in_range(ssa, group, n_group))
        return -1;
    double vert;
    return lrf_forecast(ssa, group, n_group, n_forecast, NULL, &vert, output + ssa->N, output);
}

/* The recurrence of MKL/ssa_opt.h:2818-2841 over caller-provided host data. Everything here is
 * host memory by contract (an LRF and a base signal), so the h dependent dot products run on
 * the device only when a context is at hand; this entry point has none, so it runs them here. */
int ssa_opt_forecast_with_lrf(const SSA_LRF *lrf, const ssa_real *base_signal, int base_len, int n_forecast,
                              ssa_real *output)
{
    if (!lrf || !lrf->valid || !lrf->R || !base_signal || !output)
        return -1;
    const int L = lrf->L;
    if (base_len < L - 1 || n_forecast < 1)
        return -1;
    const int w = L - 1;
    double *buf = (double *)malloc(sizeof(double) * (size_t)(w + n_forecast));
    if (!buf)
        return -1;
    for (int i = 0; i < w; i++)
        buf[i] = base_signal[base_len - w + i];
    for (int h = 0; h < n_forecast; h++)
    {
        double f = 0.0;
        for (int j = 0; j < w; j++)
            f += lrf->R[j] * buf[h + j];
        buf[w + h] = f;
        output[h] = f;
    }
    free(buf);
    return 0;
}

/* ---- getters (MKL/ssa_opt.h:3086-3145) -------------------------------------------------- */

int ssa_opt_get_trend(const SSA_Opt *ssa, ssa_real *output)
{
    int group[] = {0};
    return ssa_opt_reconstruct(ssa, group, 1, output);
}

int ssa_opt_get_noise(const SSA_Opt *ssa, int noise_start, ssa_real *output)
{
    if (!ssa || !ssa->decomposed || noise_start < 0)
        return -1;
    int n_noise = ssa->n_components - noise_start;
    if (n_noise <= 0)
    {
        memset(output, 0, sizeof(double) * ssa->N);
        return 0;
    }
    int *group = (int *)malloc(sizeof(int) * n_noise);
    if (!group)
        return -1;
    for (int i = 0; i < n_noise; i++)
        group[i] = noise_start + i;
    int ret = ssa_opt_reconstruct(ssa, group, n_noise, output);
    free(group);
    return ret;
}

ssa_real ssa_opt_variance_explained(const SSA_Opt *ssa, int start, int end)
{
    if (!ssa || !ssa->decomposed || start < 0 || ssa->total_variance <= 0)
        return 0.0;
    if (end < 0 || end >= ssa->n_components)
        end = ssa->n_components - 1;
    double sum = 0;
    for (int i = start; i <= end; i++)
        sum += ssa->eigenvalues[i];
    return sum / ssa->total_variance;
}

int ssa_opt_get_singular_values(const SSA_Opt *ssa, ssa_real *output, int max_n)
{
    if (!ssa || !ssa->decomposed || !output)
        return -1;
    int n = imin(max_n, ssa->n_components);
    memcpy(output, ssa->sigma, sizeof(double) * n);
    return n;
}

int ssa_opt_get_eigenvalues(const SSA_Opt *ssa, ssa_real *output, int max_n)
{
    if (!ssa || !ssa->decomposed || !output)
        return -1;
    int n = imin(max_n, ssa->n_components);
    memcpy(output, ssa->eigenvalues, sizeof(double) * n);
    return n;
}

ssa_real ssa_opt_get_total_variance(const SSA_Opt *ssa)
{
    if (!ssa || !ssa->decomposed)
        return 0.0;
    return ssa->total_variance;
}

/* ---- component statistics and periodic pairs (MKL/ssa_opt.h:2634-2756) ------------------ */

/* Statistics for choosing the signal rank (outputs as MKL/ssa_opt.h:2634-2695 defines them):
 *   singular_values: the decomposition's sigma;  log_sv[i] = ln(sigma_i + 1e-300);
 *   gaps[i] (i < n-1): the drop ratio sigma_i / (sigma_{i+1} + 1e-300) between neighbours;
 *   cumulative_var[i]: share of total_variance held by components 0..i;
 *   second_diff[i]: curvature of the log spectrum, log_sv[i-1] - 2 log_sv[i] + log_sv[i+1],
 *                   0 at both ends;
 *   suggested_signal: 1 + the first position of the largest drop ratio; gap_threshold: that ratio.
 * The five arrays share one allocation (released by ssa_opt_component_stats_free). -1 when not
 * decomposed or fewer than two components. */
int ssa_opt_component_stats(const SSA_Opt *ssa, SSA_ComponentStats *stats)
{
    if (!ssa || !stats || !ssa->decomposed || ssa->n_components < 2)
        return -1;
    const int n = ssa->n_components;
    double *arena = (double *)malloc(sizeof(double) * (size_t)(5 * n - 1));
    if (!arena)
        return -1;
    memset(stats, 0, sizeof(*stats));
    stats->n = n;
    stats->singular_values = arena;
    stats->log_sv = arena + n;
    stats->cumulative_var = arena + 2 * n;
    stats->second_diff = arena + 3 * n;
    stats->gaps = arena + 4 * n;
    const double *sv = ssa->sigma;
    double held = 0.0;
    int widest = 0;
    for (int i = 0; i < n; i++) {
        stats->singular_values[i] = sv[i];
        stats->log_sv[i] = log(sv[i] + 1e-300);
        held += ssa->eigenvalues[i];
        stats->cumulative_var[i] = held / ssa->total_variance;
        if (i + 1 < n) {
            stats->gaps[i] = sv[i] / (sv[i + 1] + 1e-300);
            if (stats->gaps[i] > stats->gaps[widest])
                widest = i;
        }
    }
    for (int i = 0; i < n; i++) {
        const int interior = i > 0 && i < n - 1;
        stats->second_diff[i] =
            interior ? (stats->log_sv[i - 1] + stats->log_sv[i + 1]) - 2.0 * stats->log_sv[i] : 0.0;
    }
    stats->suggested_signal = widest + 1;
    stats->gap_threshold = stats->gaps[widest];
    return 0;
}

void ssa_opt_component_stats_free(SSA_ComponentStats *stats)
{
    if (!stats)
        return;
    free(stats->singular_values); /* the one allocation behind all five arrays */
    memset(stats, 0, sizeof(*stats));
}

int ssa_opt_find_periodic_pairs(const SSA_Opt *ssa, int *pairs, int max_pairs, ssa_real sv_tol,
                                ssa_real wcorr_thresh)
{
    if (!ssa || !ssa->decomposed || !pairs || max_pairs < 1)
        return 0;
    if (sv_tol <= 0)
        sv_tol = 0.1;
    if (wcorr_thresh <= 0)
        wcorr_thresh = 0.5;
    const int n = ssa->n_components;
    double *W = (double *)malloc(sizeof(double) * n * n);
    char *used = (char *)calloc((size_t)n, 1);
    if (!W || !used || ssa_opt_wcorr_matrix(ssa, W) != 0)
    {
        free(W);
        free(used);
        return 0;
    }
    int n_pairs = 0;
    for (int i = 0; i < n - 1 && n_pairs < max_pairs; i++)
    {
        if (used[i])
            continue;
        for (int j = i + 1; j < n && n_pairs < max_pairs; j++)
        {
            if (used[j])
                continue;
            double sv_ratio = ssa->sigma[j] / (ssa->sigma[i] + 1e-300);
            if (fabs(1.0 - sv_ratio) > sv_tol)
                continue;
            if (fabs(W[i * n + j]) < wcorr_thresh)
                continue;
            pairs[2 * n_pairs] = i;
            pairs[2 * n_pairs + 1] = j;
            used[i] = used[j] = 1;
            n_pairs++;
            break;
        }
    }
    free(W);
    free(used);
    return n_pairs;
}

/* ---- V-forecast (MKL/ssa_opt.h:2906-3084) ------------------------------------------------
 * The reference's V-forecast projects the last L-1 values on every group eigenvector per step,
 *   x_new = sum_g pi_g (U_trunc,g . z) / (1 - nu^2),   pi_g = U[L-1, g],  nu^2 = sum_g pi_g^2,
 * which is R . z with R = U_trunc pi / (1 - nu^2), the LRF of the same group: the same numbers
 * as the R-forecast up to rounding. Here the projection is folded into R once on the device
 * (FP64, k_lrf) and each step is one length-(L-1) dot product instead of n_group of them.
 * Errors as the reference: -1 for an index outside the decomposition or nu^2 >= 1 - 1e-10. */

int ssa_opt_vforecast(const SSA_Opt *ssa, const int *group, int n_group, int n_forecast, ssa_real *output)
{
    if (!ssa || !ssa->decomposed || !group || !output || n_group < 1 || n_forecast < 1)
        return -1;
    if (!group_in_range(ssa, group, n_group))
        return -1;
    double vert;
    return lrf_forecast(ssa, group, n_group, n_forecast, NULL, &vert, output, NULL);
}

/* Reconstruction of the group in output[0, N), the forecast in output[N, N + n_forecast). */
int ssa_opt_vforecast_full(const SSA_Opt *ssa, const int *group, int n_group, int n_forecast, ssa_real *output)
{
    if (!ssa || !ssa->decomposed || !group || !output || n_group < 1 || n_forecast < 1)
        return -1;
    if (!group_in_range(ssa, group, n_group))
        return -1;
    double vert;
    return lrf_forecast(ssa, group, n_group, n_forecast, NULL, &vert, output + ssa->N, output);
}

/* The recurrence started from the last L-1 values of a caller-supplied base signal
 * (base_len >= L - 1) instead of the group's reconstruction. */
int ssa_opt_vforecast_fast(const SSA_Opt *ssa, const int *group, int n_group, const ssa_real *base_signal,
                           int base_len, int n_forecast, ssa_real *output)
{
    if (!ssa || !ssa->decomposed || !group || !base_signal || !output)
        return -1;
    if (n_group < 1 || n_forecast < 1 || base_len < ssa->L - 1)
        return -1;
    if (!group_in_range(ssa, group, n_group))
        return -1;
    double vert;
    return lrf_forecast_from(ssa, group, n_group, n_forecast, NULL, &vert, output, NULL,
                             base_signal + (base_len - (ssa->L - 1)));
}

/* ---- out-of-scope symbols kept for the wrapper's optional bindings ---------------------- */

/* ---- ESPRIT (MKL/ssa_opt.h:4304-4558) -----------------------------------------------------
 * The shift-invariance least squares U_up Z = U_down (U_up / U_down: rows 0..L-2 / 1..L-1 of
 * the selected eigenvectors) is solved through its normal equations: the two k x k cross Grams
 * come from the device (FP64 products of the FP32 factors, k_xgram over the factor block and its
 * one-row-shifted view), and since U has orthonormal columns U_up^T U_up = I - pi pi^T (pi: last
 * row) is well conditioned unless the group is nearly vertical, where the reference's QR solve
 * is ill-posed too. The k x k solve and eigenvalues run in FP64 on the host. */

/* Eigenvalues of a real n x n matrix (row-major a, overwritten): Householder reduction to upper
 * Hessenberg form, then Francis double-shift QR steps on the active window with deflation when a
 * subdiagonal falls below eps times its diagonal neighbours, 1x1 and 2x2 blocks read off in closed
 * form (Golub & Van Loan, Matrix Computations, Algorithms 7.4.2, 7.5.1 and 7.5.2; an exceptional
 * shift every 11th step of a stalled window). Eigenvalues are stored at their diagonal position,
 * a complex pair with the positive imaginary part first. Returns 0, or -1 without convergence
 * after 60 n steps. */
static int eig_nonsym(double *a, int n, double *wr, double *wi)
{
#define EA(i, j) a[(size_t)(i) * (size_t)n + (size_t)(j)]
    const double eps = 2.220446049250313e-16;
    double *v = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    if (!v)
        return -1;
    for (int k = 0; k + 2 < n; k++)
    {
        const int m = n - k - 1;
        double al = 0.0;
        for (int i = 0; i < m; i++)
            al += EA(k + 1 + i, k) * EA(k + 1 + i, k);
        al = sqrt(al);
        if (al == 0.0)
            continue;
        if (EA(k + 1, k) > 0.0)
            al = -al;
        for (int i = 0; i < m; i++)
            v[i] = EA(k + 1 + i, k);
        v[0] -= al;
        double vn = 0.0;
        for (int i = 0; i < m; i++)
            vn += v[i] * v[i];
        if (vn == 0.0)
            continue;
        for (int j = k; j < n; j++)
        {
            double t = 0.0;
            for (int i = 0; i < m; i++)
                t += v[i] * EA(k + 1 + i, j);
            t *= 2.0 / vn;
            for (int i = 0; i < m; i++)
                EA(k + 1 + i, j) -= t * v[i];
        }
        for (int i = 0; i < n; i++)
        {
            double t = 0.0;
            for (int j = 0; j < m; j++)
                t += EA(i, k + 1 + j) * v[j];
            t *= 2.0 / vn;
            for (int j = 0; j < m; j++)
                EA(i, k + 1 + j) -= t * v[j];
        }
        for (int i = k + 2; i < n; i++)
            EA(i, k) = 0.0;
    }
    free(v);
    double anorm = 0.0;
    for (int i = 0; i < n; i++)
        for (int j = (i > 0 ? i - 1 : 0); j < n; j++)
            anorm += fabs(EA(i, j));
    int u = n - 1, iter = 0, total = 0;
    while (u >= 0)
    {
        int l = u;
        for (; l > 0; l--)
        {
            double sc = fabs(EA(l - 1, l - 1)) + fabs(EA(l, l));
            if (sc == 0.0)
                sc = anorm;
            if (fabs(EA(l, l - 1)) <= eps * sc)
            {
                EA(l, l - 1) = 0.0;
                break;
            }
        }
        if (l == u)
        {
            wr[u] = EA(u, u);
            wi[u] = 0.0;
            u--;
            iter = 0;
            continue;
        }
        if (l == u - 1)
        {
            const double p = EA(u - 1, u - 1), q = EA(u - 1, u), r = EA(u, u - 1), d = EA(u, u);
            const double mid = 0.5 * (p + d), half = 0.5 * (p - d);
            const double disc = half * half + q * r;
            if (disc >= 0.0)
            {
                const double sq = sqrt(disc);
                const double l1 = mid + (mid >= 0.0 ? sq : -sq);
                const double l2 = l1 != 0.0 ? (p * d - q * r) / l1 : mid - sq;
                wr[u - 1] = l1;
                wr[u] = l2;
                wi[u - 1] = wi[u] = 0.0;
            }
            else
            {
                wr[u - 1] = wr[u] = mid;
                wi[u - 1] = sqrt(-disc);
                wi[u] = -wi[u - 1];
            }
            u -= 2;
            iter = 0;
            continue;
        }
        if (++total > 60 * n)
            return -1;
        iter++;
        double s, t;
        if (iter % 11 == 10)
        {
            const double w = fabs(EA(u, u - 1)) + fabs(EA(u - 1, u - 2));
            s = 1.5 * w;
            t = w * w;
        }
        else
        {
            s = EA(u - 1, u - 1) + EA(u, u);
            t = EA(u - 1, u - 1) * EA(u, u) - EA(u - 1, u) * EA(u, u - 1);
        }
        double x = EA(l, l) * EA(l, l) + EA(l, l + 1) * EA(l + 1, l) - s * EA(l, l) + t;
        double y = EA(l + 1, l) * (EA(l, l) + EA(l + 1, l + 1) - s);
        double z = EA(l + 1, l) * EA(l + 2, l + 1);
        for (int k = l; k <= u - 2; k++)
        {
            const double nrm = sqrt(x * x + y * y + z * z);
            if (nrm != 0.0)
            {
                const double beta = x > 0.0 ? -nrm : nrm;
                const double w0 = x - beta, w1 = y, w2 = z;
                const double ww = w0 * w0 + w1 * w1 + w2 * w2;
                if (ww != 0.0)
                {
                    for (int j = (k > l ? k - 1 : l); j <= u; j++)
                    {
                        const double f = 2.0 * (w0 * EA(k, j) + w1 * EA(k + 1, j) + w2 * EA(k + 2, j)) / ww;
                        EA(k, j) -= f * w0;
                        EA(k + 1, j) -= f * w1;
                        EA(k + 2, j) -= f * w2;
                    }
                    const int r1 = k + 3 < u ? k + 3 : u;
                    for (int i = l; i <= r1; i++)
                    {
                        const double f = 2.0 * (EA(i, k) * w0 + EA(i, k + 1) * w1 + EA(i, k + 2) * w2) / ww;
                        EA(i, k) -= f * w0;
                        EA(i, k + 1) -= f * w1;
                        EA(i, k + 2) -= f * w2;
                    }
                    if (k > l)
                    {
                        EA(k + 1, k - 1) = 0.0;
                        EA(k + 2, k - 1) = 0.0;
                    }
                }
            }
            x = EA(k + 1, k);
            y = EA(k + 2, k);
            if (k < u - 2)
                z = EA(k + 3, k);
        }
        const double nrm = sqrt(x * x + y * y);
        if (nrm != 0.0)
        {
            const double beta = x > 0.0 ? -nrm : nrm;
            const double w0 = x - beta, w1 = y;
            const double ww = w0 * w0 + w1 * w1;
            if (ww != 0.0)
            {
                for (int j = u - 2; j <= u; j++)
                {
                    const double f = 2.0 * (w0 * EA(u - 1, j) + w1 * EA(u, j)) / ww;
                    EA(u - 1, j) -= f * w0;
                    EA(u, j) -= f * w1;
                }
                for (int i = l; i <= u; i++)
                {
                    const double f = 2.0 * (EA(i, u - 1) * w0 + EA(i, u) * w1) / ww;
                    EA(i, u - 1) -= f * w0;
                    EA(i, u) -= f * w1;
                }
                EA(u, u - 2) = 0.0;
            }
        }
    }
#undef EA
    return 0;
}

int ssa_b200_eigvals(int n, const double *A, double *wr, double *wi)
{
    if (n < 1 || !A || !wr || !wi)
        return -1;
    double *a = (double *)malloc(sizeof(double) * (size_t)n * (size_t)n);
    if (!a)
        return -1;
    memcpy(a, A, sizeof(double) * (size_t)n * (size_t)n);
    const int rc = eig_nonsym(a, n, wr, wi);
    free(a);
    return rc;
}

int ssa_opt_parestimate(const SSA_Opt *ssa, const int *group, int n_group, SSA_ParEstimate *result)
{
    if (!ssa || !ssa->decomposed || !result)
        return -1;
    const int nc = ssa->n_components;
    const int k = (n_group > 0 && group) ? n_group : nc;
    if (k < 1 || k > nc)
        return -1;
    const int L = ssa->L;
    if (L < 3)
        return -1;
    int *idx = (int *)malloc(sizeof(int) * (size_t)k);
    if (!idx)
        return -1;
    for (int j = 0; j < k; j++)
    {
        idx[j] = (n_group > 0 && group) ? group[j] : j;
        if (idx[j] < 0 || idx[j] >= nc)
        {
            free(idx);
            return -1;
        }
    }
    struct ssa_gpu_ctx *g = ssa->gpu;
    ssa_engine *e = &g->e;
    const int m = L - 1;
    int rows = (m + 127) / 128;
    rows = ((rows + SSA_GRAM_CHUNK - 1) / SSA_GRAM_CHUNK) * SSA_GRAM_CHUNK;
    const int nch = (m + rows - 1) / rows;
    const size_t np = (size_t)nch * nc * nc;
    double *d_part = NULL, *h_part = (double *)malloc(sizeof(double) * 2 * np);
    double *G = (double *)calloc((size_t)nc * nc * 2, sizeof(double));
    double *Z = (double *)malloc(sizeof(double) * (size_t)k * k * 3);
    double *wr = (double *)malloc(sizeof(double) * (size_t)k * 2);
    int rc = !h_part || !G || !Z || !wr || ssae_dalloc(e, (void **)&d_part, sizeof(double) * 2 * np) != 0;
    if (!rc)
    {
        /* job 0: U_up^T U_up, job 1: U_up^T U_down (the same block one row further down) */
        ssa_xgram_job J[2];
        memset(J, 0, sizeof(J));
        for (int q = 0; q < 2; q++)
        {
            J[q].A = e->Y;
            J[q].B = e->Y + q;
            J[q].part = d_part + (size_t)q * np;
            J[q].lda = J[q].ldb = e->ldL;
            J[q].m = m;
            J[q].na = J[q].nb = nc;
            J[q].rows_per_cta = rows;
        }
        ssae_reset_jobs(e);
        void *d = ssae_push_jobs(e, J, sizeof(J));
        rc = !d || ssad_xgram((const ssa_xgram_job *)d, 2, nch, e->st) != 0 ||
             cudaMemcpyAsync(h_part, d_part, sizeof(double) * 2 * np, cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
             sync_ok(g) != 0;
    }
    ssae_dfree(e, d_part);
    if (!rc)
    {
        for (int q = 0; q < 2; q++)
            for (int c = 0; c < nch; c++)
                for (size_t t = 0; t < (size_t)nc * nc; t++)
                    G[(size_t)q * nc * nc + t] += h_part[(size_t)q * np + (size_t)c * nc * nc + t];
        /* the group's k x k blocks: Gs = U_up^T U_up, Cs = U_up^T U_down (row-major) */
        double *Gs = Z + (size_t)k * k, *Cs = Gs + (size_t)k * k;
        for (int a = 0; a < k; a++)
            for (int b = 0; b < k; b++)
            {
                Gs[a * k + b] = G[(size_t)idx[a] * nc + idx[b]];
                Cs[a * k + b] = G[(size_t)nc * nc + (size_t)idx[a] * nc + idx[b]];
            }
        /* Cholesky Gs = R^T R (upper R in place), then Z = R^-1 R^-T Cs */
        for (int j = 0; j < k && !rc; j++)
        {
            double d = Gs[j * k + j];
            for (int p = 0; p < j; p++)
                d -= Gs[p * k + j] * Gs[p * k + j];
            if (!(d > 0.0))
            {
                rc = 1;
                break;
            }
            d = sqrt(d);
            Gs[j * k + j] = d;
            for (int c = j + 1; c < k; c++)
            {
                double t = Gs[j * k + c];
                for (int p = 0; p < j; p++)
                    t -= Gs[p * k + j] * Gs[p * k + c];
                Gs[j * k + c] = t / d;
            }
        }
        if (!rc)
        {
            for (int c = 0; c < k; c++)
            {
                /* solve R^T y = Cs[:, c], then R z = y */
                for (int i = 0; i < k; i++)
                {
                    double t = Cs[i * k + c];
                    for (int p = 0; p < i; p++)
                        t -= Gs[p * k + i] * Z[p * k + c];
                    Z[i * k + c] = t / Gs[i * k + i];
                }
                for (int i = k - 1; i >= 0; i--)
                {
                    double t = Z[i * k + c];
                    for (int p = i + 1; p < k; p++)
                        t -= Gs[i * k + p] * Z[p * k + c];
                    Z[i * k + c] = t / Gs[i * k + i];
                }
            }
            rc = eig_nonsym(Z, k, wr, wr + k) != 0;
        }
    }
    if (!rc)
    {
        memset(result, 0, sizeof(*result));
        result->periods = (double *)malloc(sizeof(double) * (size_t)k);
        result->frequencies = (double *)malloc(sizeof(double) * (size_t)k);
        result->moduli = (double *)malloc(sizeof(double) * (size_t)k);
        result->rates = (double *)malloc(sizeof(double) * (size_t)k);
        result->n_components = k;
        if (!result->periods || !result->frequencies || !result->moduli || !result->rates)
        {
            ssa_opt_parestimate_free(result);
            rc = 1;
        }
        for (int i = 0; i < k && !rc; i++)
        {
            const double re = wr[i], im = wr[k + i];
            const double mod = sqrt(re * re + im * im);
            const double freq = atan2(im, re) / (2.0 * M_PI);
            result->moduli[i] = mod;
            result->rates[i] = mod > 1e-12 ? log(mod) : -30.0;
            result->frequencies[i] = freq;
            result->periods[i] = fabs(freq) > 1e-12 ? 1.0 / fabs(freq) : INFINITY;
        }
    }
    free(idx);
    free(h_part);
    free(G);
    free(Z);
    free(wr);
    return rc ? -1 : 0;
}
void ssa_opt_parestimate_free(SSA_ParEstimate *result)
{
    if (!result)
        return;
    free(result->periods);
    free(result->frequencies);
    free(result->moduli);
    free(result->rates);
    memset(result, 0, sizeof(*result));
}

/* ---- MKL tuning exports of MKL/py/ssa_wrapper.c:47-123 ---------------------------------- */
int ssa_mkl_init(int verbose)
{
    (void)verbose;
    return 0;
}
int ssa_mkl_init_14900kf(int verbose)
{
    (void)verbose;
    return 0;
}
int ssa_mkl_init_generic(int verbose)
{
    (void)verbose;
    return 0;
}
void ssa_mkl_set_threads(int n) { (void)n; }
int ssa_mkl_get_threads(void) { return 1; }
void ssa_mkl_get_cpu_info(int *p_cores, int *e_cores, int *is_hybrid, int *has_avx512)
{
    if (p_cores)
        *p_cores = 0;
    if (e_cores)
        *e_cores = 0;
    if (is_hybrid)
        *is_hybrid = 0;
    if (has_avx512)
        *has_avx512 = 0;
}
void ssa_mkl_disable_affinity(void) {}

/* ---- matvec diagnostics (reference static helpers MKL/ssa_opt.h:871-903) ----------------- */
static int matvec_dev(SSA_Opt *ssa, const double *in, double *out, int adjoint)
{
    if (!ssa || !ssa->initialized || !in || !out)
        return -1;
    struct ssa_gpu_ctx *g = ssa->gpu;
    ssa_engine *e = &g->e;
    const int nin = adjoint ? ssa->L : ssa->K, nout = adjoint ? ssa->K : ssa->L;
    float *dst_in = adjoint ? e->Y : e->Z, *src_out = adjoint ? e->Z : e->Y;
    if (ensure_stage(g, (size_t)(ssa->L > ssa->K ? ssa->L : ssa->K)) != 0)
        return -1;
    ssae_reset_jobs(e);
    for (int i = 0; i < nin; i++)
        g->h_stage[i] = (float)in[i];
    if (cudaMemcpyAsync(dst_in, g->h_stage, sizeof(float) * nin, cudaMemcpyHostToDevice, e->st) != cudaSuccess ||
        ssae_matvec(e, 1, adjoint) != 0 ||
        cudaMemcpyAsync(g->h_stage, src_out, sizeof(float) * nout, cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
        sync_ok(g) != 0)
        return -1;
    for (int i = 0; i < nout; i++)
        out[i] = (double)g->h_stage[i];
    /* the matvec overwrote the first columns of the factor buffers */
    ssa->decomposed = false;
    g->spectra_valid = 0;
    g->wcorr_valid = 0;
    return 0;
}

int ssa_opt_hankel_matvec_dev(SSA_Opt *ssa, const double *v, double *y) { return matvec_dev(ssa, v, y, 0); }
int ssa_opt_hankel_matvec_T_dev(SSA_Opt *ssa, const double *u, double *z) { return matvec_dev(ssa, u, z, 1); }
void ssa_opt_hankel_matvec(SSA_Opt *ssa, const double *v, double *y) { (void)matvec_dev(ssa, v, y, 0); }
void ssa_opt_hankel_matvec_T(SSA_Opt *ssa, const double *u, double *z) { (void)matvec_dev(ssa, u, z, 1); }

int ssa_opt_copy_factors(const SSA_Opt *ssa, double *U, double *V)
{
    if (!ssa || !ssa->decomposed)
        return -1;
    const int k = ssa->n_components;
    if (U)
        memcpy(U, ssa->U, sizeof(double) * (size_t)ssa->L * k);
    if (V)
        memcpy(V, ssa->V, sizeof(double) * (size_t)ssa->K * k);
    return k;
}

/* ---- Cadzow iterations (MKL/ssa_opt.h:3165-3442) --------------------------------------------
 * The signal stays on the device for the whole loop: each iteration decomposes the context's
 * current signal, reconstructs the leading `rank` components into g->d_out and reduces
 * ||y_new - y|| on the device; the host reads back two doubles per iteration for the stopping
 * test. The reference picks the randomized branch when rank + 8 < min(L, K) / 2 (:3212) and the
 * block method (block size min(rank, 16), 3 iterations) otherwise or when the randomized one
 * fails (:3213-3232). */

static int cadzow_use_randomized(int rank, int L, int K) { return rank + 8 < imin(L, K) / 2; }

/* Decompose the current device signal (spectrum already in e->X) to `rank` components and
 * reconstruct them into g->d_out; waits for the device. 0 on success, -1 on a launch error, 1
 * when the decomposition reported a failure status. */
static int cadzow_project(SSA_Opt *ssa, int rank, int randomized, unsigned long long seed, int *k_out)
{
    struct ssa_gpu_ctx *g = ssa->gpu;
    ssa_engine *e = &g->e;
    const int L = ssa->L, K = ssa->K;
    int k;
    g->spectra_valid = 0;
    g->wcorr_valid = 0;
    if (randomized)
    {
        const int kp = imin(rank + 8, imin(L, K));
        k = imin(rank, kp);
        if (kp > e->kp || ssae_decompose(e, 1, kp, k, 0, NULL, 0, seed) != 0)
            return -1;
    }
    else
    {
        k = imin(rank, imin(L, K));
        if (k > e->k || ssae_decompose_block(e, 1, k, imin(rank, 16), 3, NULL, K, seed) != 0)
            return -1;
    }
    if (sync_ok(g) != 0)
        return -1;
    if (check_status(g) != 0)
        return 1;
    if (ssae_spectra(e, 1, k) != 0 || ssae_recon_group(e, 0, k, g->d_group, rank, g->d_out) != 0)
        return -1;
    g->spectra_valid = 1;
    ssa->n_components = k;
    *k_out = k;
    return 0;
}

static int cadzow_setup(struct ssa_gpu_ctx *g, int rank, double **d_aux, size_t aux_doubles)
{
    int *grp = (int *)malloc(sizeof(int) * rank);
    if (!grp)
        return -1;
    for (int i = 0; i < rank; i++)
        grp[i] = i;
    int rc = ensure_group(g, grp, rank);
    rc |= sync_ok(g);
    free(grp);
    if (rc || ssae_dalloc(&g->e, (void **)d_aux, sizeof(double) * aux_doubles) != 0)
        return -1;
    return cudaMemsetAsync(*d_aux, 0, sizeof(double) * aux_doubles, g->e.st) == cudaSuccess ? 0 : -1;
}

/* The Cadzow loop on x. With y1 given (the rank-`rank` projection of x, e.g. from factors the
 * caller keeps), that projection counts as the first iteration: its difference to x is measured
 * and the loop continues from it, so the result equals the plain loop's whenever y1 equals what
 * the first decomposition would give. */
static int cadzow_run_from(const double *x, const double *y1, int N, int L, int rank, int max_iter, double tol,
                           double alpha, double *output, SSA_CadzowResult *result);

static int cadzow_run(const double *x, int N, int L, int rank, int max_iter, double tol, double alpha,
                      double *output, SSA_CadzowResult *result)
{
    return cadzow_run_from(x, NULL, N, L, rank, max_iter, tol, alpha, output, result);
}

int ssab_cadzow_from(const double *x, const double *y1, int N, int L, int rank, int max_iter, double tol,
                     double *output, SSA_CadzowResult *result)
{
    return cadzow_run_from(x, y1, N, L, rank, max_iter, tol, 1.0, output, result);
}

static int cadzow_run_from(const double *x, const double *y1, int N, int L, int rank, int max_iter, double tol,
                           double alpha, double *output, SSA_CadzowResult *result)
{
    if (!x || !output || N < 4 || L < 2 || L > N - 1 || rank < 1 || max_iter < 1)
        return -1;
    const int K = N - L + 1;
    if (imin(rank, imin(L, K)) > SSA_MAX_KP)
        return -1;
    SSA_Opt ssa;
    if (ssa_opt_init(&ssa, x, N, L) != 0)
        return -1;
    struct ssa_gpu_ctx *g = ssa.gpu;
    ssa_engine *e = &g->e;
    double *d_aux = NULL; /* diff^2, |y|^2, then the input signal when blending */
    const int blend = alpha < 1.0;
    if (cadzow_setup(g, rank, &d_aux, 2 + (blend ? (size_t)N : 0)) != 0)
    {
        ssa_opt_free(&ssa);
        return -1;
    }
    double ynorm = 0.0;
    for (int i = 0; i < N; i++)
        ynorm += x[i] * x[i];
    ynorm = sqrt(ynorm);
    if (ynorm < 1e-15)
        ynorm = 1.0;
    int rc = 0, iter, k = 0;
    double diff = 0.0;
    int converged = 0;
    if (blend)
        rc |= cudaMemcpyAsync(d_aux + 2, e->x64, sizeof(double) * N, cudaMemcpyDeviceToDevice, e->st) != cudaSuccess;
    const int randomized = cadzow_use_randomized(rank, L, K);
    for (iter = 0; iter < max_iter && !rc; iter++)
    {
        ssae_reset_jobs(e);
        if (iter > 0 && ssae_signal_spectrum(e, e->x64, 1) != 0)
        {
            rc = -1;
            break;
        }
        if (iter == 0 && y1)
        {
            /* the given first projection stands in for the first decomposition */
            if (cudaMemcpyAsync(g->d_out, y1, sizeof(double) * N, cudaMemcpyHostToDevice, e->st) != cudaSuccess)
            {
                rc = -1;
                break;
            }
        }
        else
        {
            /* every iteration runs in a freshly initialised context in the reference, whose
             * generator restarts: the same seed each time */
            int pr = 1;
            if (randomized)
                pr = cadzow_project(&ssa, rank, 1, SSA_DEFAULT_SEED, &k);
            if (pr == 1)
                pr = cadzow_project(&ssa, rank, 0, SSA_DEFAULT_SEED ^ 0xB10CB10CB10CB10CULL, &k);
            if (pr != 0)
            {
                rc = -1;
                break;
            }
        }
        double h[2];
        if (ssad_diffnorm(g->d_out, e->x64, N, d_aux, e->st) != 0 ||
            cudaMemcpyAsync(e->x64, g->d_out, sizeof(double) * N, cudaMemcpyDeviceToDevice, e->st) != cudaSuccess ||
            cudaMemcpyAsync(h, d_aux, sizeof(double) * 2, cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
            sync_ok(g) != 0)
        {
            rc = -1;
            break;
        }
        diff = sqrt(h[0]) / ynorm;
        if (diff < tol)
        {
            converged = 1;
            iter++;
            break;
        }
    }
    if (!rc && blend &&
        ssad_axpby(e->x64, d_aux + 2, e->x64, alpha, 1.0 - alpha, N, e->st) != 0)
        rc = -1;
    if (!rc && (cudaMemcpyAsync(output, e->x64, sizeof(double) * N, cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
                sync_ok(g) != 0))
        rc = -1;
    ssae_dfree(&g->e, d_aux);
    ssa_opt_free(&ssa);
    if (rc)
        return -1;
    if (result)
    {
        result->iterations = iter;
        result->final_diff = diff;
        result->converged = converged ? 1.0 : 0.0;
    }
    return iter;
}

int ssa_opt_cadzow(const ssa_real *x, int N, int L, int rank, int max_iter, ssa_real tol, ssa_real *output,
                   SSA_CadzowResult *result)
{
    return cadzow_run(x, N, L, rank, max_iter, tol, 1.0, output, result);
}

/* output = alpha * cadzow(x) + (1 - alpha) * x (MKL/ssa_opt.h:3294-3315), blended on the device. */
int ssa_opt_cadzow_weighted(const ssa_real *x, int N, int L, int rank, int max_iter, ssa_real tol, ssa_real alpha,
                            ssa_real *output, SSA_CadzowResult *result)
{
    if (alpha <= 0.0 || alpha > 1.0)
        return -1;
    return cadzow_run(x, N, L, rank, max_iter, tol, alpha, output, result);
}

/* In-place variant (MKL/ssa_opt.h:3319-3442): iterates on the context's own signal. The first
 * reconstruction sets the norm for the relative difference; later ones are compared with the
 * previous reconstruction; the signal is replaced by the reconstruction except after the last
 * iteration. The randomized branch needs a prepared context with room for rank + 8 columns and
 * draws a new test matrix per call, like the reference's generator stream. On return the context
 * holds the last decomposition (host fields mirrored). */
int ssa_opt_cadzow_inplace(SSA_Opt *ssa, int rank, int max_iter, ssa_real tol, SSA_CadzowResult *result)
{
    if (!ssa || !ssa->initialized || rank < 1 || max_iter < 1)
        return -1;
    const int N = ssa->N, L = ssa->L, K = ssa->K;
    if (imin(rank, imin(L, K)) > SSA_MAX_KP)
        return -1;
    struct ssa_gpu_ctx *g = ssa->gpu;
    ssa_engine *e = &g->e;
    double *d_aux = NULL; /* diff^2, |y|^2, previous reconstruction (N) */
    ssae_reset_jobs(e);
    if (cadzow_setup(g, rank, &d_aux, 2 + (size_t)N) != 0)
        return -1;
    double *d_prev = d_aux + 2;
    double y_norm = 1.0, diff = 0.0;
    int converged = 0, iter, rc = 0, k = 0;
    for (iter = 0; iter < max_iter; iter++)
    {
        ssae_reset_jobs(e);
        const int randomized = cadzow_use_randomized(rank, L, K);
        ssa_opt_free_cached_ffts(ssa);
        ssa->decomposed = false;
        ssa->n_components = 0;
        ssa->total_variance = 0.0;
        int pr = 1;
        if (randomized && ssa->prepared && rank + 8 <= ssa->prepared_kp)
        {
            const unsigned long long seed = SSA_DEFAULT_SEED + 0x100000000ULL * (unsigned long long)ssa->rng_calls;
            ssa->rng_calls++;
            pr = cadzow_project(ssa, rank, 1, seed, &k);
        }
        if (pr == 1)
        {
            const unsigned long long seed =
                (SSA_DEFAULT_SEED + 0x100000000ULL * (unsigned long long)ssa->rng_calls) ^ 0xB10CB10CB10CB10CULL;
            ssa->rng_calls++;
            pr = cadzow_project(ssa, rank, 0, seed, &k);
        }
        if (pr != 0)
        {
            rc = -1;
            break;
        }
        double h[2];
        if (ssad_diffnorm(g->d_out, d_prev, N, d_aux, e->st) != 0 ||
            cudaMemcpyAsync(d_prev, g->d_out, sizeof(double) * N, cudaMemcpyDeviceToDevice, e->st) != cudaSuccess ||
            cudaMemcpyAsync(h, d_aux, sizeof(double) * 2, cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
            sync_ok(g) != 0)
        {
            rc = -1;
            break;
        }
        if (iter == 0)
        {
            y_norm = sqrt(h[1]);
            if (y_norm < 1e-15)
                y_norm = 1.0;
        }
        else
        {
            diff = sqrt(h[0]) / y_norm;
            if (diff < tol)
            {
                converged = 1;
                iter++;
                break;
            }
        }
        if (iter < max_iter - 1)
        {
            /* the decomposition's factors stay in the engine; only the signal and its spectrum
             * change (the engine keeps them apart) */
            if (cudaMemcpyAsync(e->x64, g->d_out, sizeof(double) * N, cudaMemcpyDeviceToDevice, e->st) !=
                    cudaSuccess ||
                ssae_signal_spectrum(e, e->x64, 1) != 0)
            {
                rc = -1;
                break;
            }
        }
    }
    ssae_dfree(&g->e, d_aux);
    if (rc)
        return -1;
    /* mirror the last decomposition and the current signal's spectrum */
    if (alloc_results(ssa, k) != 0)
        return -1;
    ssa->n_components = k;
    if (mirror_results(ssa, k) != 0 || mirror_spectrum(ssa) != 0)
        return -1;
    ssa->decomposed = true;
    if (result)
    {
        result->iterations = iter;
        result->final_diff = diff;
        result->converged = converged ? 1.0 : 0.0;
    }
    return iter;
}

/* ---- gap filling (MKL/ssa_opt.h:3440-3878) ------------------------------------------------
 * Missing values are NaN. Both forms modify x in place at the gap positions only. */

/* Gaps start as the straight line between their valid neighbours (one neighbour: that value;
 * none: 0), point j of a gap of length n at fraction (j + 1) / (n + 1) (a single point: 1/2). */
static void gap_linear_start(double *x, const unsigned char *gap, int N)
{
    int i = 0;
    while (i < N)
    {
        if (!gap[i])
        {
            i++;
            continue;
        }
        const int a = i;
        while (i < N && gap[i])
            i++;
        const int n = i - a;
        const double lv = a > 0 ? x[a - 1] : (i < N ? x[i] : 0.0);
        const double rv = i < N ? x[i] : lv;
        for (int j = 0; j < n; j++)
        {
            const double t = n > 1 ? (double)(j + 1) / (double)(n + 1) : 0.5;
            x[a + j] = lv + t * (rv - lv);
        }
    }
}

static int gap_mask(const double *x, int N, unsigned char **gap)
{
    *gap = (unsigned char *)calloc((size_t)N, 1);
    if (!*gap)
        return -1;
    int n = 0;
    for (int i = 0; i < N; i++)
        if (isnan(x[i]))
        {
            (*gap)[i] = 1;
            n++;
        }
    return n;
}

/* Iterative form: each iteration reconstructs the current signal from its leading `rank`
 * components (randomized, q = 0, oversampling 8, as the reference's freshly initialised context
 * per iteration: the same test matrix every time) and writes the reconstruction into the gaps,
 * until the relative change of the gap values drops below tol. Device-resident: the signal stays
 * in HBM, each iteration reads back two sums. Returns 0 (iterations etc. in result) or -1. */
int ssa_opt_gapfill(ssa_real *x, int N, int L, int rank, int max_iter, ssa_real tol, SSA_GapFillResult *result)
{
    if (!x || N < 4 || L < 2 || L > N - 1 || rank < 1)
        return -1;
    unsigned char *gap = NULL;
    const int n_gaps = gap_mask(x, N, &gap);
    if (n_gaps < 0)
        return -1;
    if (n_gaps == 0)
    {
        free(gap);
        if (result)
        {
            result->iterations = 0;
            result->final_diff = 0.0;
            result->converged = 1;
            result->n_gaps = 0;
        }
        return 0;
    }
    const int K = N - L + 1;
    if (N - n_gaps < L + rank || imin(rank + 8, imin(L, K)) > SSA_MAX_KP)
    {
        free(gap);
        return -1;
    }
    int *idx = (int *)malloc(sizeof(int) * (size_t)n_gaps);
    if (!idx)
    {
        free(gap);
        return -1;
    }
    for (int i = 0, j = 0; i < N; i++)
        if (gap[i])
            idx[j++] = i;
    gap_linear_start(x, gap, N);
    free(gap);
    SSA_Opt ssa;
    if (ssa_opt_init(&ssa, x, N, L) != 0)
    {
        free(idx);
        return -1;
    }
    struct ssa_gpu_ctx *g = ssa.gpu;
    ssa_engine *e = &g->e;
    double *d_aux = NULL; /* two sums, then the gap indices */
    int rc = cadzow_setup(g, rank, &d_aux, 2 + ((size_t)n_gaps + 1) / 2);
    int *d_idx = d_aux ? (int *)(d_aux + 2) : NULL;
    if (!rc && cudaMemcpyAsync(d_idx, idx, sizeof(int) * (size_t)n_gaps, cudaMemcpyHostToDevice, e->st) != cudaSuccess)
        rc = -1;
    free(idx);
    int iter = 0, converged = 0, k = 0;
    double diff = 1e10;
    for (iter = 0; iter < max_iter && !rc; iter++)
    {
        ssae_reset_jobs(e);
        if (iter > 0 && ssae_signal_spectrum(e, e->x64, 1) != 0)
        {
            rc = -1;
            break;
        }
        if (cadzow_project(&ssa, rank, 1, SSA_DEFAULT_SEED, &k) != 0)
        {
            rc = -1;
            break;
        }
        double h[2];
        if (ssad_gapupdate(e->x64, g->d_out, d_idx, n_gaps, d_aux, e->st) != 0 ||
            cudaMemcpyAsync(h, d_aux, sizeof(double) * 2, cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
            sync_ok(g) != 0)
        {
            rc = -1;
            break;
        }
        diff = h[1] > 1e-12 ? sqrt(h[0] / h[1]) : sqrt(h[0]);
        if (diff < tol)
        {
            converged = 1;
            iter++;
            break;
        }
    }
    if (!rc && (cudaMemcpyAsync(x, e->x64, sizeof(double) * (size_t)N, cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
                sync_ok(g) != 0))
        rc = -1;
    ssae_dfree(&g->e, d_aux);
    ssa_opt_free(&ssa);
    if (rc)
        return -1;
    if (result)
    {
        result->iterations = iter;
        result->final_diff = diff;
        result->converged = converged;
        result->n_gaps = n_gaps;
    }
    return 0;
}

/* h-step forecast of the leading `rank` components of data[0, n) (randomized, q = 0,
 * oversampling 8, a fresh context): a malloc'd array, or NULL when the segment cannot be
 * decomposed or forecast. */
static double *segment_forecast(const double *data, int n, int L, int rank, const int *group, int h)
{
    SSA_Opt s;
    if (ssa_opt_init(&s, data, n, L) != 0)
        return NULL;
    double *f = NULL;
    if (ssa_opt_prepare(&s, rank, 8) == 0 && ssa_opt_decompose_randomized(&s, rank, 8) == 0)
    {
        f = (double *)malloc(sizeof(double) * (size_t)h);
        if (f && ssa_opt_forecast(&s, group, imin(rank, s.n_components), h, f) != 0)
        {
            free(f);
            f = NULL;
        }
    }
    ssa_opt_free(&s);
    return f;
}

/* Single-pass form: every gap run (left to right, earlier runs already filled) is filled from a
 * forecast of the valid segment before it and a forecast of the reversed segment after it (each
 * when at least L + rank long), weighted linearly towards the nearer side; with neither, the mean
 * of the neighbouring values. A forecast that cannot be computed counts as absent, and so does a
 * segment that still holds a later, unfilled gap (the reference decomposes the NaNs there). */
int ssa_opt_gapfill_simple(ssa_real *x, int N, int L, int rank, SSA_GapFillResult *result)
{
    if (!x || N < 4 || L < 2 || L > N - 1 || rank < 1)
        return -1;
    unsigned char *gap = NULL;
    const int n_gaps = gap_mask(x, N, &gap);
    if (n_gaps < 0)
        return -1;
    int *group = (int *)malloc(sizeof(int) * (size_t)rank);
    double *rev = (double *)malloc(sizeof(double) * (size_t)N);
    if (!group || !rev)
    {
        free(gap);
        free(group);
        free(rev);
        return -1;
    }
    for (int i = 0; i < rank; i++)
        group[i] = i;
    int i = 0;
    while (i < N)
    {
        if (!gap[i])
        {
            i++;
            continue;
        }
        const int a = i;
        while (i < N && gap[i])
            i++;
        const int glen = i - a, right_len = N - i;
        double *fl = a >= L + rank ? segment_forecast(x, a, L, rank, group, glen) : NULL;
        double *fr = NULL;
        int right_clean = right_len >= L + rank;
        for (int j = i; j < N && right_clean; j++)
            right_clean = !gap[j];
        if (right_clean)
        {
            for (int j = 0; j < right_len; j++)
                rev[j] = x[N - 1 - j];
            fr = segment_forecast(rev, right_len, L, rank, group, glen);
        }
        for (int j = 0; j < glen; j++)
        {
            double v = 0.0, w = 0.0;
            if (fl)
            {
                const double wl = (double)(glen - j) / glen;
                v += wl * fl[j];
                w += wl;
            }
            if (fr)
            {
                const double wr = (double)(j + 1) / glen;
                v += wr * fr[glen - 1 - j]; /* the backcast runs from the right end */
                w += wr;
            }
            if (w > 0.0)
                x[a + j] = v / w;
            else
            {
                const double lv = a > 0 ? x[a - 1] : 0.0;
                const double rv = i < N ? x[i] : lv;
                x[a + j] = 0.5 * (lv + rv);
            }
        }
        free(fl);
        free(fr);
    }
    free(gap);
    free(group);
    free(rev);
    if (result)
    {
        result->iterations = 1;
        result->final_diff = 0.0;
        result->converged = 1;
        result->n_gaps = n_gaps;
    }
    return 0;
}


void ssa_b200_set_wcorr_tensor_cores(int on) { ssad_set_wcorr_tc(on ? 1 : 0); }
int ssa_b200_wcorr_tensor_cores(void) { return ssad_wcorr_tc() != 0; }
int ssa_b200_set_wcorr_gram(int mode)
{
    if (mode < 0 || mode > 3)
        return -1;
    ssad_set_wcorr_tc(mode);
    return 0;
}
int ssa_b200_wcorr_gram(void) { return ssad_wcorr_tc(); }
void ssa_b200_set_rowmul_tensor_cores(int on) { ssad_set_rowmul_tc(on); }
int ssa_b200_rowmul_tensor_cores(void) { return ssad_rowmul_tc_on(); }

/* ---- library information ----------------------------------------------------------------- */
unsigned long long ssa_b200_kernel_launches(void) { return ssad_launch_count(); }
int ssa_b200_device_checks(unsigned int *out5, int reset) { return ssad_read_checks(out5, reset) == 0 ? 0 : -1; }
int ssa_b200_sizeof_ssa_opt(void) { return (int)sizeof(SSA_Opt); }
