/*
 * MSSA entry points (reference MKL/ssa_opt.h:3880-4283) on the device engine. The M channels of
 * one instance are the engine's series: each has its own signal spectrum and its L-row block
 * of the stacked left vectors; the right vectors V are shared. Host layout of the results is the
 * reference's: U is (M L) x k column-major with channel m's block in rows m L .. m L + L - 1.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "ssa_engine.h"
#include "../../include/ssa_opt.h"

struct mssa_gpu_ctx
{
    ssa_engine e;
    int ok;
    int k_cap;
    int spectra_valid;
    float *h_stage;
    size_t stage_cap;
    int *d_group;
    int group_cap;
    double *d_out;       /* N */
    double *d_contrib;   /* M * k */
};

static int imin(int a, int b) { return a < b ? a : b; }

static void mgpu_free(struct mssa_gpu_ctx *g)
{
    if (!g)
        return;
    if (g->ok)
        ssae_destroy(&g->e);
    if (g->h_stage)
        cudaFreeHost(g->h_stage);
    if (g->d_group)
        cudaFree(g->d_group);
    if (g->d_out)
        cudaFree(g->d_out);
    if (g->d_contrib)
        cudaFree(g->d_contrib);
    free(g);
}

static int mstage(struct mssa_gpu_ctx *g, size_t floats)
{
    if (floats <= g->stage_cap)
        return 0;
    if (g->h_stage)
        cudaFreeHost(g->h_stage);
    g->h_stage = NULL;
    g->stage_cap = 0;
    if (cudaMallocHost((void **)&g->h_stage, floats * sizeof(float)) != cudaSuccess)
        return -1;
    g->stage_cap = floats;
    return 0;
}

void mssa_opt_free(MSSA_Opt *mssa)
{
    if (!mssa)
        return;
    mgpu_free(mssa->gpu);
    free(mssa->U);
    free(mssa->V);
    free(mssa->sigma);
    free(mssa->eigenvalues);
    free(mssa->inv_diag_count);
    memset(mssa, 0, sizeof(*mssa));
}

int mssa_opt_init(MSSA_Opt *mssa, const ssa_real *X, int M, int N, int L)
{
    if (!mssa || !X || M < 1 || N < 4 || L < 2 || L > N - 1)
        return -1;
    memset(mssa, 0, sizeof(*mssa));
    const int logh = ssad_logh_for(N);
    if (logh > SSA_MAX_LOGH_ALL)
        return -1;
    mssa->M = M;
    mssa->N = N;
    mssa->L = L;
    mssa->K = N - L + 1;
    mssa->fft_len = 2 << logh;
    mssa->r2c_len = (1 << logh) + 1;
    struct mssa_gpu_ctx *g = (struct mssa_gpu_ctx *)calloc(1, sizeof(*g));
    if (!g)
        return -1;
    mssa->gpu = g;
    const int kp = imin(SSA_MAX_KP, imin(M * L, mssa->K));
    if (ssae_create(&g->e, M, N, L, kp, kp, NULL) != 0)
    {
        free(g);
        mssa->gpu = NULL;
        return -1;
    }
    g->ok = 1;
    g->k_cap = kp;
    mssa->inv_diag_count = (double *)malloc(sizeof(double) * N);
    if (!mssa->inv_diag_count || cudaMalloc((void **)&g->d_out, sizeof(double) * N) != cudaSuccess ||
        cudaMalloc((void **)&g->d_contrib, sizeof(double) * (size_t)M * kp) != cudaSuccess)
    {
        mssa_opt_free(mssa);
        return -1;
    }
    for (int t = 0; t < N; t++)
    {
        int c = imin(imin(t + 1, L), imin(mssa->K, N - t));
        mssa->inv_diag_count[t] = c > 0 ? 1.0 / c : 0.0;
    }
    ssae_reset_jobs(&g->e);
    if (cudaMemcpyAsync(g->e.x64, X, sizeof(double) * (size_t)M * N, cudaMemcpyHostToDevice, g->e.st) != cudaSuccess ||
        ssae_signal_spectrum(&g->e, g->e.x64, M) != 0 || cudaStreamSynchronize(g->e.st) != cudaSuccess)
    {
        mssa_opt_free(mssa);
        return -1;
    }
    mssa->initialized = true;
    return 0;
}

static int mssa_decompose_impl(MSSA_Opt *mssa, int k, int oversampling, int q, const double *Omega)
{
    if (!mssa || !mssa->initialized || k < 1 || q < 0)
        return -1;
    const int M = mssa->M, L = mssa->L, K = mssa->K, ML = M * L;
    const int p = oversampling <= 0 ? 8 : oversampling;
    int kp = imin(k + p, imin(ML, K));
    k = imin(k, kp);
    struct mssa_gpu_ctx *g = mssa->gpu;
    if (kp > g->k_cap)
        return -1;
    ssa_engine *e = &g->e;
    ssae_reset_jobs(e);
    mssa->decomposed = false;
    g->spectra_valid = 0;
    free(mssa->U);
    free(mssa->V);
    free(mssa->sigma);
    free(mssa->eigenvalues);
    mssa->U = (double *)calloc((size_t)ML * k, sizeof(double));
    mssa->V = (double *)calloc((size_t)K * k, sizeof(double));
    mssa->sigma = (double *)calloc((size_t)k, sizeof(double));
    mssa->eigenvalues = (double *)calloc((size_t)k, sizeof(double));
    if (!mssa->U || !mssa->V || !mssa->sigma || !mssa->eigenvalues)
        return -1;
    mssa->n_components = k;
    int rc = 0;
    if (Omega)
    {
        if (mstage(g, (size_t)K * kp) != 0)
            return -1;
        for (size_t i = 0; i < (size_t)K * kp; i++)
            g->h_stage[i] = (float)Omega[i];
        rc |= cudaMemcpy2DAsync(e->Z, sizeof(float) * e->ldK, g->h_stage, sizeof(float) * K, sizeof(float) * K, kp,
                                cudaMemcpyHostToDevice, e->st) != cudaSuccess;
        rc |= ssae_mssa_decompose(e, M, kp, k, q, e->Z, 0) != 0;
    }
    else
    {
        const unsigned long long seed = (42ULL + 0x100000000ULL * (unsigned long long)mssa->rng_calls) ^
                                        0x4D55535341ULL;
        mssa->rng_calls++;
        rc |= ssae_mssa_decompose(e, M, kp, k, q, NULL, seed) != 0;
    }
    if (rc || cudaStreamSynchronize(e->st) != cudaSuccess)
        return -1;
    int st = 0;
    if (cudaMemcpy(&st, e->status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess || st != 0)
        return -1;
    /* mirror U (per channel), V, sigma */
    if (mstage(g, (size_t)(L > K ? L : K) * k) != 0)
        return -1;
    const size_t sY = (size_t)e->ldL * e->kp;
    for (int m = 0; m < M; m++)
    {
        if (cudaMemcpy2D(g->h_stage, sizeof(float) * L, e->Y + (size_t)m * sY, sizeof(float) * e->ldL,
                         sizeof(float) * L, k, cudaMemcpyDeviceToHost) != cudaSuccess)
            return -1;
        for (int i = 0; i < k; i++)
            for (int r = 0; r < L; r++)
                mssa->U[(size_t)i * ML + (size_t)m * L + r] = (double)g->h_stage[(size_t)i * L + r];
    }
    if (cudaMemcpy2D(g->h_stage, sizeof(float) * K, e->Z, sizeof(float) * e->ldK, sizeof(float) * K, k,
                     cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(mssa->sigma, e->sigma, sizeof(double) * k, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    for (size_t i = 0; i < (size_t)K * k; i++)
        mssa->V[i] = (double)g->h_stage[i];
    mssa->total_variance = 0.0;
    for (int i = 0; i < k; i++)
    {
        mssa->eigenvalues[i] = mssa->sigma[i] * mssa->sigma[i];
        mssa->total_variance += mssa->eigenvalues[i];
    }
    mssa->decomposed = true;
    return 0;
}

int mssa_opt_decompose(MSSA_Opt *mssa, int k, int oversampling)
{
    return mssa_decompose_impl(mssa, k, oversampling, 0, NULL);
}

int mssa_opt_decompose_ex(MSSA_Opt *mssa, int k, int oversampling, int power_iters, const double *Omega)
{
    return mssa_decompose_impl(mssa, k, oversampling, power_iters, Omega);
}

/* Reconstruction of channel m from the cached spectra of sigma_i u_i^(m) and v_i into g->d_out. */
static int mssa_recon_dev(const MSSA_Opt *mssa, int m, const int *group, int n_group)
{
    struct mssa_gpu_ctx *g = mssa->gpu;
    ssa_engine *e = &g->e;
    if (!g->spectra_valid)
    {
        if (ssae_spectra(e, mssa->M, mssa->n_components) != 0)
            return -1;
        g->spectra_valid = 1;
    }
    if (n_group > g->group_cap)
    {
        if (g->d_group)
            cudaFree(g->d_group);
        g->d_group = NULL;
        g->group_cap = 0;
        if (cudaMalloc((void **)&g->d_group, sizeof(int) * (n_group < 64 ? 64 : n_group)) != cudaSuccess)
            return -1;
        g->group_cap = n_group < 64 ? 64 : n_group;
    }
    if (cudaMemcpyAsync(g->d_group, group, sizeof(int) * n_group, cudaMemcpyHostToDevice, e->st) != cudaSuccess)
        return -1;
    return ssae_recon_group(e, m, mssa->n_components, g->d_group, n_group, g->d_out) != 0 ? -1 : 0;
}

int mssa_opt_reconstruct(const MSSA_Opt *mssa, int series_idx, const int *group, int n_group, ssa_real *output)
{
    if (!mssa || !mssa->decomposed || !group || !output || n_group < 1 || series_idx < 0 ||
        series_idx >= mssa->M)
        return -1;
    struct mssa_gpu_ctx *g = mssa->gpu;
    ssae_reset_jobs(&g->e);
    if (mssa_recon_dev(mssa, series_idx, group, n_group) != 0 ||
        cudaMemcpyAsync(output, g->d_out, sizeof(double) * mssa->N, cudaMemcpyDeviceToHost, g->e.st) != cudaSuccess ||
        cudaStreamSynchronize(g->e.st) != cudaSuccess)
        return -1;
    return 0;
}

int mssa_opt_reconstruct_all(const MSSA_Opt *mssa, const int *group, int n_group, ssa_real *output)
{
    if (!mssa || !mssa->decomposed || !group || !output || n_group < 1)
        return -1;
    for (int m = 0; m < mssa->M; m++)
        if (mssa_opt_reconstruct(mssa, m, group, n_group, output + (size_t)m * mssa->N) != 0)
            return -1;
    return 0;
}

/* contributions[m * k + i] = ||U^(m)[:, i]||^2 (MKL/ssa_opt.h:4255-4271), computed on the device. */
int mssa_opt_series_contributions(const MSSA_Opt *mssa, ssa_real *contributions)
{
    if (!mssa || !mssa->decomposed || !contributions)
        return -1;
    struct mssa_gpu_ctx *g = mssa->gpu;
    ssa_engine *e = &g->e;
    const int k = mssa->n_components;
    ssae_reset_jobs(e);
    if (ssad_colnorm2(e->Y, (long long)e->ldL * e->kp, e->ldL, mssa->L, k, mssa->M, g->d_contrib, e->st) != 0 ||
        cudaMemcpyAsync(contributions, g->d_contrib, sizeof(double) * (size_t)mssa->M * k, cudaMemcpyDeviceToHost,
                        e->st) != cudaSuccess ||
        cudaStreamSynchronize(e->st) != cudaSuccess)
        return -1;
    return 0;
}

ssa_real mssa_opt_variance_explained(const MSSA_Opt *mssa, int start, int end)
{
    if (!mssa || !mssa->decomposed || start < 0 || mssa->total_variance <= 0)
        return 0.0;
    if (end < 0 || end >= mssa->n_components)
        end = mssa->n_components - 1;
    double sum = 0;
    for (int i = start; i <= end; i++)
        sum += mssa->eigenvalues[i];
    return sum / mssa->total_variance;
}

int mssa_opt_copy_factors(const MSSA_Opt *mssa, double *U, double *V, double *sigma)
{
    if (!mssa || !mssa->decomposed)
        return -1;
    const int k = mssa->n_components;
    if (U)
        memcpy(U, mssa->U, sizeof(double) * (size_t)mssa->M * mssa->L * k);
    if (V)
        memcpy(V, mssa->V, sizeof(double) * (size_t)mssa->K * k);
    if (sigma)
        memcpy(sigma, mssa->sigma, sizeof(double) * k);
    return k;
}
