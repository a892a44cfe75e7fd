/*
 * Batched multichannel SSA with Cadzow iterations: I independent instances of M channels of
 * length N (the stacked (M L) x K trajectory operator of MKL/ssa_opt.h:3880-4283 per instance),
 * all on one device engine whose series are the I M channels.
 *
 * One Cadzow iteration of every instance at once (the multivariate form of the reference's
 * ssa_opt_cadzow loop, MKL/ssa_opt.h:3165-3290, which the reference has for one channel only):
 *   signal spectra of the current channels -> block power of each stacked operator
 *   (ssae_mssa_batch_decompose: one block of kp = k + p columns, q iterations) -> V_i and sigma_i
 *   handed to the instance's channels -> spectra of sigma_c u_c and v_c -> reconstruction of
 *   components 0 .. k-1 of every channel (edge anti-diagonals exact) -> the change
 *   ||y_new - y|| of every channel -> the reconstructions become the channels.
 * The test matrix of instance i is the device generator's with seed ^ golden (i + 1), the same in
 * every iteration (the reference restarts its generator in every iteration's fresh context).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "ssa_engine.h"
#include "../../include/ssa_opt.h"

struct ssa_mbatch
{
    ssa_engine e;
    int live;
    int I, M, N, L, K, k, kp, q;
    double *d_y, *d_ynew; /* I M x N current and new channels */
    double *d_norm;       /* I M x 2: ||x_c||^2 of the input */
    double *d_diff;       /* iterations x I M x 2 */
    int *d_group;         /* 0 .. k-1 */
    int iters_cap;
    ssa_copy_seg *h_segs; /* broadcast of V_i and sigma_i to the channels */
};

#define CKM(x)                 \
    do                         \
    {                          \
        if ((x) != cudaSuccess) \
            return -1;         \
    } while (0)

static int imin(int a, int b) { return a < b ? a : b; }

void ssa_mbatch_destroy(ssa_mbatch *mb)
{
    if (!mb)
        return;
    if (mb->live)
    {
        cudaStreamSynchronize(mb->e.st);
        ssae_destroy(&mb->e);
    }
    void *d[] = {mb->d_y, mb->d_ynew, mb->d_norm, mb->d_diff, mb->d_group};
    for (size_t i = 0; i < sizeof(d) / sizeof(d[0]); i++)
        if (d[i])
            cudaFree(d[i]);
    if (mb->h_segs)
        cudaFreeHost(mb->h_segs);
    free(mb);
}

int ssa_mbatch_create(ssa_mbatch **out, int I, int M, int N, int L, int k, int oversampling, int power_iters)
{
    if (!out || I < 1 || M < 1 || N < 4 || L < 2 || L > N - 1 || k < 1 || power_iters < 0)
        return -1;
    *out = NULL;
    const int K = N - L + 1;
    const int p = oversampling <= 0 ? 8 : oversampling;
    const int kp = imin(k + p, imin(M * L, K));
    if (kp > SSA_MAX_KP || ssad_logh_for(N) > SSA_MAX_LOGH_ALL)
        return -1;
    ssa_mbatch *mb = (ssa_mbatch *)calloc(1, sizeof(*mb));
    if (!mb)
        return -1;
    mb->I = I;
    mb->M = M;
    mb->N = N;
    mb->L = L;
    mb->K = K;
    mb->k = imin(k, kp);
    mb->kp = kp;
    mb->q = power_iters;
    const int B = I * M;
    int *grp = (int *)malloc(sizeof(int) * (size_t)mb->k);
    if (!grp || ssae_create(&mb->e, B, N, L, kp, mb->k, NULL) != 0)
    {
        free(grp);
        free(mb);
        return -1;
    }
    mb->live = 1;
    for (int i = 0; i < mb->k; i++)
        grp[i] = i;
    const size_t nseg = (size_t)B * 2;
    const int rc = cudaMalloc((void **)&mb->d_y, sizeof(double) * (size_t)B * N) != cudaSuccess ||
                   cudaMalloc((void **)&mb->d_ynew, sizeof(double) * (size_t)B * N) != cudaSuccess ||
                   cudaMalloc((void **)&mb->d_norm, sizeof(double) * 2 * (size_t)B) != cudaSuccess ||
                   cudaMalloc((void **)&mb->d_group, sizeof(int) * (size_t)mb->k) != cudaSuccess ||
                   cudaMemcpy(mb->d_group, grp, sizeof(int) * (size_t)mb->k, cudaMemcpyHostToDevice) != cudaSuccess ||
                   cudaMallocHost((void **)&mb->h_segs, sizeof(ssa_copy_seg) * nseg) != cudaSuccess;
    free(grp);
    if (rc)
    {
        ssa_mbatch_destroy(mb);
        return -1;
    }
    *out = mb;
    return 0;
}

/* Instance i's V (channel i M's Z slot, first k columns) and sigma into its other channels. */
static int broadcast(ssa_mbatch *mb)
{
    ssa_engine *e = &mb->e;
    const size_t sZ = (size_t)e->ldK * e->kp;
    size_t n = 0;
    for (int i = 0; i < mb->I; i++)
        for (int m = 1; m < mb->M; m++)
        {
            const int c0 = i * mb->M, c = c0 + m;
            /* V: ldK k floats (ldK a multiple of 4) copied as doubles */
            mb->h_segs[n].src = (const double *)(e->Z + (size_t)c0 * sZ);
            mb->h_segs[n].dst = (double *)(e->Z + (size_t)c * sZ);
            mb->h_segs[n].n = (long long)e->ldK * mb->k / 2;
            n++;
            mb->h_segs[n].src = e->sigma + (size_t)c0 * e->k;
            mb->h_segs[n].dst = e->sigma + (size_t)c * e->k;
            mb->h_segs[n].n = mb->k;
            n++;
        }
    if (!n)
        return 0;
    void *d = ssae_push_jobs(e, mb->h_segs, sizeof(ssa_copy_seg) * n);
    if (!d)
        return -1;
    return ssad_copy_segments((const ssa_copy_seg *)d, (int)n, e->st) != 0 ? -1 : 0;
}

/* Reconstruction of components 0 .. k-1 of every channel into d_ynew. */
static int recon_all(ssa_mbatch *mb)
{
    ssa_engine *e = &mb->e;
    const int B = mb->I * mb->M;
    ssa_recon_job *jobs = (ssa_recon_job *)calloc((size_t)B, sizeof(ssa_recon_job));
    if (!jobs)
        return -1;
    for (int c = 0; c < B; c++)
    {
        ssa_recon_job *J = &jobs[c];
        J->Us = e->Us + (size_t)c * e->k * e->ldS;
        J->Vs = e->Vs + (size_t)c * e->k * e->ldS;
        J->U = e->Y + (size_t)c * e->ldL * e->kp;
        J->V = e->Z + (size_t)c * e->ldK * e->kp;
        J->ldU = e->ldL;
        J->ldV = e->ldK;
        J->sigma = e->sigma + (size_t)c * e->k;
        J->group = mb->d_group;
        J->out64 = mb->d_ynew + (size_t)c * mb->N;
        J->ld_spec = e->ldS;
        J->n_group = mb->k;
        J->k = mb->k;
        J->N = mb->N;
        J->L = mb->L;
        J->K = mb->K;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_recon_job) * B);
    free(jobs);
    if (!d)
        return -1;
    return ssad_recon((const ssa_recon_job *)d, B, e->logh, e->st) != 0 ? -1 : 0;
}

int ssa_mbatch_run_device(ssa_mbatch *mb, const double *d_X, int iters, uint64_t seed, double *d_out,
                          double *d_sigma)
{
    if (!mb || !d_X || iters < 1)
        return -1;
    ssa_engine *e = &mb->e;
    const int B = mb->I * mb->M, N = mb->N;
    ssae_reset_jobs(e);
    if (iters > mb->iters_cap)
    {
        if (mb->d_diff)
            cudaFree(mb->d_diff);
        mb->d_diff = NULL;
        mb->iters_cap = 0;
        CKM(cudaMalloc((void **)&mb->d_diff, sizeof(double) * 2 * (size_t)B * iters));
        mb->iters_cap = iters;
    }
    /* the job tables of every stage of every iteration stay in the arena until the run ends */
    const size_t per_iter = (size_t)B * (3 * sizeof(ssa_col_job) + 2 * sizeof(ssa_gram_job) + 2 * sizeof(ssa_rowmul_job) +
                                         sizeof(ssa_recon_job) + 2 * sizeof(ssa_copy_seg)) * (size_t)(6 + 4 * mb->q) +
                            (1 << 16);
    if (ssae_grow_arena(e, per_iter * (size_t)iters) != 0)
        return -1;
    CKM(cudaMemcpyAsync(mb->d_y, d_X, sizeof(double) * (size_t)B * N, cudaMemcpyDeviceToDevice, e->st));
    if (ssad_diffnorm_batch(mb->d_y, mb->d_y, N, B, mb->d_norm, e->st) != 0)
        return -1;
    for (int t = 0; t < iters; t++)
    {
        if (ssae_signal_spectrum(e, mb->d_y, B) != 0 ||
            ssae_mssa_batch_decompose(e, mb->I, mb->M, mb->kp, mb->k, mb->q, seed) != 0 || broadcast(mb) != 0 ||
            ssae_spectra(e, B, mb->k) != 0 || recon_all(mb) != 0 ||
            ssad_diffnorm_batch(mb->d_ynew, mb->d_y, N, B, mb->d_diff + (size_t)t * 2 * B, e->st) != 0)
            return -1;
        double *tmp = mb->d_y;
        mb->d_y = mb->d_ynew;
        mb->d_ynew = tmp;
    }
    if (d_out)
        CKM(cudaMemcpyAsync(d_out, mb->d_y, sizeof(double) * (size_t)B * N, cudaMemcpyDeviceToDevice, e->st));
    if (d_sigma)
        CKM(cudaMemcpy2DAsync(d_sigma, sizeof(double) * mb->k, e->sigma, sizeof(double) * (size_t)mb->M * e->k,
                              sizeof(double) * mb->k, (size_t)mb->I, cudaMemcpyDeviceToDevice, e->st));
    return 0;
}

int ssa_mbatch_sync(ssa_mbatch *mb)
{
    if (!mb || cudaStreamSynchronize(mb->e.st) != cudaSuccess)
        return -1;
    int *st = (int *)malloc(sizeof(int) * (size_t)mb->I);
    if (!st)
        return -1;
    int bad = cudaMemcpy(st, mb->e.status, sizeof(int) * (size_t)mb->I, cudaMemcpyDeviceToHost) != cudaSuccess;
    for (int i = 0; i < mb->I && !bad; i++)
        bad = st[i] != 0;
    free(st);
    return bad ? -1 : 0;
}

int ssa_mbatch_diffs(ssa_mbatch *mb, int iters, double *diff)
{
    if (!mb || !diff || iters < 1 || iters > mb->iters_cap)
        return -1;
    const int B = mb->I * mb->M;
    double *h = (double *)malloc(sizeof(double) * 2 * (size_t)B * (iters + 1));
    if (!h)
        return -1;
    if (cudaStreamSynchronize(mb->e.st) != cudaSuccess ||
        cudaMemcpy(h, mb->d_norm, sizeof(double) * 2 * (size_t)B, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(h + 2 * (size_t)B, mb->d_diff, sizeof(double) * 2 * (size_t)B * iters, cudaMemcpyDeviceToHost) !=
            cudaSuccess)
    {
        free(h);
        return -1;
    }
    for (int i = 0; i < mb->I; i++)
    {
        double x2 = 0.0;
        for (int m = 0; m < mb->M; m++)
            x2 += h[2 * (size_t)(i * mb->M + m) + 1];
        const double xn = x2 > 1e-30 ? sqrt(x2) : 1.0;
        for (int t = 0; t < iters; t++)
        {
            double d2 = 0.0;
            for (int m = 0; m < mb->M; m++)
                d2 += h[2 * (size_t)B * (t + 1) + 2 * (size_t)(i * mb->M + m)];
            diff[(size_t)i * iters + t] = sqrt(d2) / xn;
        }
    }
    free(h);
    return 0;
}

int ssa_mbatch_run(ssa_mbatch *mb, const double *X, int iters, uint64_t seed, double *out, double *sigma, double *diff)
{
    if (!mb || !X || iters < 1)
        return -1;
    const int B = mb->I * mb->M;
    const size_t nx = (size_t)B * mb->N;
    double *d_x = NULL, *d_out = NULL, *d_sig = NULL;
    int rc = -1;
    if (cudaMalloc((void **)&d_x, sizeof(double) * nx) == cudaSuccess &&
        cudaMalloc((void **)&d_out, sizeof(double) * nx) == cudaSuccess &&
        cudaMalloc((void **)&d_sig, sizeof(double) * (size_t)mb->I * mb->k) == cudaSuccess &&
        cudaMemcpyAsync(d_x, X, sizeof(double) * nx, cudaMemcpyHostToDevice, mb->e.st) == cudaSuccess &&
        ssa_mbatch_run_device(mb, d_x, iters, seed, d_out, d_sig) == 0 && ssa_mbatch_sync(mb) == 0 &&
        (!out || cudaMemcpy(out, d_out, sizeof(double) * nx, cudaMemcpyDeviceToHost) == cudaSuccess) &&
        (!sigma || cudaMemcpy(sigma, d_sig, sizeof(double) * (size_t)mb->I * mb->k, cudaMemcpyDeviceToHost) ==
                       cudaSuccess) &&
        (!diff || ssa_mbatch_diffs(mb, iters, diff) == 0))
        rc = 0;
    cudaStreamSynchronize(mb->e.st);
    cudaFree(d_x);
    cudaFree(d_out);
    cudaFree(d_sig);
    return rc;
}

int ssa_mbatch_dims(const ssa_mbatch *mb, int *k, int *kp)
{
    if (!mb)
        return -1;
    if (k)
        *k = mb->k;
    if (kp)
        *kp = mb->kp;
    return 0;
}

void *ssa_mbatch_stream(const ssa_mbatch *mb) { return mb ? (void *)mb->e.st : NULL; }
