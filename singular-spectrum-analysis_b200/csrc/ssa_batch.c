/*
 * Batched hot path: B series of identical (N, L) through the device engine in one launch per
 * stage (decomposition, elementary reconstructions, W-correlation, group sums).
 */
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "ssa_engine.h"
#include "../../include/ssa_opt.h"

struct ssa_batch
{
    ssa_engine e;
    int k, kp, q, n_groups, total_idx;
    int *d_group_idx, *d_group_off;
    double *d_groups;   /* B x n_groups x N */
    double *d_x;        /* staging for host runs */
    int last_nb;
};

static int imin(int a, int b) { return a < b ? a : b; }

void ssa_batch_destroy(ssa_batch *b)
{
    if (!b)
        return;
    ssae_destroy(&b->e);
    if (b->d_group_idx)
        cudaFree(b->d_group_idx);
    if (b->d_group_off)
        cudaFree(b->d_group_off);
    if (b->d_groups)
        cudaFree(b->d_groups);
    if (b->d_x)
        cudaFree(b->d_x);
    free(b);
}

int ssa_batch_create(ssa_batch **out, int max_series, int N, int L, int k, int oversampling, int power_iters,
                     const int *group_idx, const int *group_sizes, int n_groups)
{
    if (!out || max_series < 1 || N < 4 || L < 2 || L > N - 1 || k < 1 || power_iters < 0 || n_groups < 0)
        return -1;
    *out = NULL;
    const int K = N - L + 1;
    const int p = oversampling <= 0 ? 8 : oversampling;
    const int kp = imin(k + p, imin(L, K));
    k = imin(k, kp);
    if (kp > SSA_MAX_KP)
        return -1;
    ssa_batch *b = (ssa_batch *)calloc(1, sizeof(*b));
    if (!b)
        return -1;
    if (ssae_create(&b->e, max_series, N, L, kp, k, NULL) != 0)
    {
        free(b);
        return -1;
    }
    b->k = k;
    b->kp = kp;
    b->q = power_iters;
    b->n_groups = n_groups;
    if (ssae_ensure_recon(&b->e) != 0)
    {
        ssa_batch_destroy(b);
        return -1;
    }
    if (n_groups > 0)
    {
        int *off = (int *)malloc(sizeof(int) * (n_groups + 1));
        if (!off)
        {
            ssa_batch_destroy(b);
            return -1;
        }
        off[0] = 0;
        for (int g = 0; g < n_groups; g++)
            off[g + 1] = off[g] + (group_sizes[g] > 0 ? group_sizes[g] : 0);
        b->total_idx = off[n_groups];
        int rc = 0;
        rc |= cudaMalloc((void **)&b->d_group_off, sizeof(int) * (n_groups + 1)) != cudaSuccess;
        rc |= cudaMalloc((void **)&b->d_group_idx, sizeof(int) * (b->total_idx > 0 ? b->total_idx : 1)) != cudaSuccess;
        rc |= cudaMalloc((void **)&b->d_groups, sizeof(double) * (size_t)max_series * n_groups * N) != cudaSuccess;
        if (!rc)
        {
            rc |= cudaMemcpy(b->d_group_off, off, sizeof(int) * (n_groups + 1), cudaMemcpyHostToDevice) != cudaSuccess;
            if (b->total_idx > 0)
                rc |= cudaMemcpy(b->d_group_idx, group_idx, sizeof(int) * b->total_idx, cudaMemcpyHostToDevice) !=
                      cudaSuccess;
        }
        free(off);
        if (rc)
        {
            ssa_batch_destroy(b);
            return -1;
        }
    }
    *out = b;
    return 0;
}

int ssa_batch_run_device(ssa_batch *b, const double *d_x, int B, uint64_t seed)
{
    if (!b || !d_x || B < 1 || B > b->e.B)
        return -1;
    ssa_engine *e = &b->e;
    ssae_reset_jobs(e);
    b->last_nb = B;
    if (ssae_signal_spectrum(e, d_x, B) != 0)
        return -1;
    if (ssae_decompose(e, B, b->kp, b->k, b->q, NULL, 0, (unsigned long long)seed) != 0)
        return -1;
    if (ssae_elem_recon(e, B, b->k) != 0)
        return -1;
    if (ssae_wcorr(e, B, b->k) != 0)
        return -1;
    if (b->n_groups > 0)
    {
        ssa_gsum_job J;
        memset(&J, 0, sizeof(J));
        J.recon = e->recon;
        J.ld_recon = e->ldN;
        J.recon_series = (long long)e->k * e->ldN;
        J.group_idx = b->d_group_idx;
        J.group_off = b->d_group_off;
        J.out = b->d_groups;
        J.out_series = (long long)b->n_groups * e->N;
        J.n_groups = b->n_groups;
        J.N = e->N;
        J.k = b->k;
        J.B = B;
        ssae_prof_begin(e, SSAK_GSUM);
        int rc = ssad_group_sum(J, e->st);
        ssae_prof_end(e);
        if (rc != 0)
            return -1;
    }
    return 0;
}

int ssa_batch_sync(ssa_batch *b)
{
    if (!b)
        return -1;
    if (cudaStreamSynchronize(b->e.st) != cudaSuccess)
        return -1;
    const int nb = b->last_nb;
    if (nb <= 0)
        return 0;
    int *st = (int *)malloc(sizeof(int) * nb);
    if (!st)
        return -1;
    int rc = cudaMemcpy(st, b->e.status, sizeof(int) * nb, cudaMemcpyDeviceToHost) != cudaSuccess;
    for (int s = 0; s < nb && !rc; s++)
        if (st[s] != 0)
            rc = 1;
    free(st);
    return rc ? -1 : 0;
}

int ssa_batch_run(ssa_batch *b, const double *x, int B, uint64_t seed, double *sigma, double *W, double *groups)
{
    if (!b || !x || B < 1 || B > b->e.B)
        return -1;
    ssa_engine *e = &b->e;
    if (!b->d_x && cudaMalloc((void **)&b->d_x, sizeof(double) * (size_t)e->B * e->N) != cudaSuccess)
        return -1;
    ssae_reset_jobs(e);
    if (cudaMemcpyAsync(b->d_x, x, sizeof(double) * (size_t)B * e->N, cudaMemcpyHostToDevice, e->st) != cudaSuccess)
        return -1;
    if (ssa_batch_run_device(b, b->d_x, B, seed) != 0)
        return -1;
    /* copy (not reset) — jobs of this run are in flight until the stream drains */
    if (sigma && cudaMemcpyAsync(sigma, e->sigma, sizeof(double) * (size_t)B * b->k, cudaMemcpyDeviceToHost,
                                 e->st) != cudaSuccess)
        return -1;
    if (W && cudaMemcpyAsync(W, e->W, sizeof(double) * (size_t)B * b->k * b->k, cudaMemcpyDeviceToHost, e->st) !=
                 cudaSuccess)
        return -1;
    if (groups && b->n_groups > 0 &&
        cudaMemcpyAsync(groups, b->d_groups, sizeof(double) * (size_t)B * b->n_groups * e->N,
                        cudaMemcpyDeviceToHost, e->st) != cudaSuccess)
        return -1;
    return ssa_batch_sync(b);
}

int ssa_batch_device_results(const ssa_batch *b, ssa_batch_results *out)
{
    if (!b || !out)
        return -1;
    out->sigma = b->e.sigma;
    out->W = b->e.W;
    out->groups = b->d_groups;
    out->recon = b->e.recon;
    out->ld_recon = b->e.ldN;
    out->status = b->e.status;
    out->stream = (void *)b->e.st;
    return 0;
}

int ssa_batch_set_profiling(ssa_batch *b, int on)
{
    if (!b)
        return -1;
    return ssae_set_profiling(&b->e, on);
}

int ssa_batch_profile(ssa_batch *b, double *ms, long long *launches, int nkinds)
{
    if (!b || !ms || !launches)
        return -1;
    if (ssae_prof_collect(&b->e) != 0)
        return -1;
    const int n = nkinds < SSAK_NKINDS ? nkinds : SSAK_NKINDS;
    for (int k = 0; k < n; k++)
    {
        ms[k] = b->e.prof_ms[k];
        launches[k] = b->e.prof_n[k];
    }
    return SSAK_NKINDS;
}

int ssa_batch_status(ssa_batch *b, int *status, int n)
{
    if (!b || !status || n < 1 || n > b->e.B)
        return -1;
    if (cudaStreamSynchronize(b->e.st) != cudaSuccess)
        return -1;
    return cudaMemcpy(status, b->e.status, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}
