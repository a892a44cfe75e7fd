/*
 * Device pipeline for B series (see ssa_engine.h). Every stage fills job tables on the host,
 * stages them through pinned memory into device memory on the engine's stream and launches
 * one kernel per stage over all series. Nothing here computes numbers on the CPU.
 *
 * Randomized decomposition (reference MKL/ssa_opt.h:1685-1763, plus q power iterations):
 *   Y = H Omega;
 *   repeat q times: Q = CholQR(Y); Z = H^T Q; Z = CholQR(Z); Y = H Z;
 *   Q = CholQR2(Y);
 *   B = H^T Q; B^T B = Z_r Lambda Z_r^T (FP64 Jacobi); sigma = sqrt(Lambda);
 *   U = Q Z_r[:, :k], V = B Z_r[:, :k] Sigma^{-1}, signs so that sum_i U[i, j] >= 0.
 */
#include "ssa_engine.h"

#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define CK(x)                              \
    do                                     \
    {                                      \
        int _e = (int)(x);                 \
        if (_e != 0)                       \
            return _e;                     \
    } while (0)

static long long round4(long long v) { return (v + 3) & ~3LL; }
static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

static int gram_rows(int m, int B)
{
    /* Aim for about 1184 CTAs (eight per SM) over all series (latency hiding when a launch holds
     * few series). */
    int target = 1184 / (B > 0 ? B : 1);
    if (target < 1)
        target = 1;
    int rows = (m + target - 1) / target;
    rows = ((rows + SSA_GRAM_CHUNK - 1) / SSA_GRAM_CHUNK) * SSA_GRAM_CHUNK;
    /* at least four staging chunks per CTA: fewer partials for the per-series kernels to sum
     * (their latency) when a launch holds few series */
    return imax(rows, 4 * SSA_GRAM_CHUNK);
}

/* ---- Context recycling ---------------------------------------------------------------------
 * A drop-in caller creates and frees a context per series (SSA(x, L) ... free), and every
 * context needs a stream, a page-locked job arena and a dozen device buffers. Created fresh,
 * that costs driver calls that synchronise the device (cudaFree, cudaFreeHost) or pin pages
 * (cudaMallocHost) on every request. With recycling on (the default), engines that own their
 * stream take it from a per-device stack of streams that earlier contexts returned, take device
 * buffers from the library's stream-ordered memory pool on that stream (freed blocks stay cached
 * in the pool) and take page-locked blocks from a per-device free list. ssa_b200_set_context_
 * recycling(0) restores plain allocation for contexts created afterwards. */
#define SSA_RECYCLE_STREAMS 64
#define SSA_RECYCLE_PINNED 16
#define SSA_RECYCLE_DEVICES 64

static pthread_mutex_t g_recycle_mu = PTHREAD_MUTEX_INITIALIZER;
static int g_recycle_on = 1;
static cudaStream_t g_free_streams[SSA_RECYCLE_DEVICES][SSA_RECYCLE_STREAMS];
static int g_n_free_streams[SSA_RECYCLE_DEVICES];
static struct
{
    void *p;
    size_t cap;
} g_free_pinned[SSA_RECYCLE_DEVICES][SSA_RECYCLE_PINNED];
static int g_n_free_pinned[SSA_RECYCLE_DEVICES];

void ssa_b200_set_context_recycling(int on)
{
    pthread_mutex_lock(&g_recycle_mu);
    g_recycle_on = on != 0;
    pthread_mutex_unlock(&g_recycle_mu);
}

int ssa_b200_context_recycling(void) { return g_recycle_on; }

static int recycle_dev(int device) { return device >= 0 && device < SSA_RECYCLE_DEVICES; }

static int stream_take(int device, cudaStream_t *st)
{
    *st = NULL;
    if (recycle_dev(device))
    {
        pthread_mutex_lock(&g_recycle_mu);
        if (g_n_free_streams[device] > 0)
            *st = g_free_streams[device][--g_n_free_streams[device]];
        pthread_mutex_unlock(&g_recycle_mu);
    }
    if (*st)
        return 0;
    return (int)cudaStreamCreateWithFlags(st, cudaStreamNonBlocking);
}

static void stream_return(int device, cudaStream_t st)
{
    int kept = 0;
    if (recycle_dev(device))
    {
        pthread_mutex_lock(&g_recycle_mu);
        if (g_n_free_streams[device] < SSA_RECYCLE_STREAMS)
        {
            g_free_streams[device][g_n_free_streams[device]++] = st;
            kept = 1;
        }
        pthread_mutex_unlock(&g_recycle_mu);
    }
    if (!kept)
        cudaStreamDestroy(st);
}

/* Smallest free page-locked block of at least `bytes` (its capacity in *cap), else a new one. */
static int pinned_take(int device, size_t bytes, void **p, size_t *cap)
{
    *p = NULL;
    if (recycle_dev(device))
    {
        pthread_mutex_lock(&g_recycle_mu);
        int best = -1;
        for (int i = 0; i < g_n_free_pinned[device]; i++)
            if (g_free_pinned[device][i].cap >= bytes &&
                (best < 0 || g_free_pinned[device][i].cap < g_free_pinned[device][best].cap))
                best = i;
        if (best >= 0)
        {
            *p = g_free_pinned[device][best].p;
            *cap = g_free_pinned[device][best].cap;
            g_free_pinned[device][best] = g_free_pinned[device][--g_n_free_pinned[device]];
        }
        pthread_mutex_unlock(&g_recycle_mu);
    }
    if (*p)
        return 0;
    *cap = bytes;
    return (int)cudaMallocHost(p, bytes);
}

/* Back to the free list (the block's users have finished with it); beyond the list's length
 * the smallest block is released. */
static void pinned_return(int device, void *p, size_t cap)
{
    void *drop = p;
    if (recycle_dev(device))
    {
        pthread_mutex_lock(&g_recycle_mu);
        if (g_n_free_pinned[device] < SSA_RECYCLE_PINNED)
        {
            g_free_pinned[device][g_n_free_pinned[device]].p = p;
            g_free_pinned[device][g_n_free_pinned[device]].cap = cap;
            g_n_free_pinned[device]++;
            drop = NULL;
        }
        else
        {
            int small = 0;
            for (int i = 1; i < SSA_RECYCLE_PINNED; i++)
                if (g_free_pinned[device][i].cap < g_free_pinned[device][small].cap)
                    small = i;
            if (g_free_pinned[device][small].cap < cap)
            {
                drop = g_free_pinned[device][small].p;
                g_free_pinned[device][small].p = p;
                g_free_pinned[device][small].cap = cap;
            }
        }
        pthread_mutex_unlock(&g_recycle_mu);
    }
    if (drop)
        cudaFreeHost(drop);
}

int ssae_dalloc(ssa_engine *e, void **p, size_t bytes)
{
    *p = NULL;
    if (bytes == 0)
        return 0;
    if (e->recycle)
    {
        cudaMemPool_t pool = ssar_pool();
        if (pool)
            return (int)cudaMallocFromPoolAsync(p, bytes, pool, e->st);
    }
    return (int)cudaMalloc(p, bytes);
}

void ssae_dfree(ssa_engine *e, void *p)
{
    if (!p)
        return;
    if (e->recycle)
        cudaFreeAsync(p, e->st);
    else
        cudaFree(p);
}

int ssae_pinned(ssa_engine *e, size_t bytes, void **p, size_t *cap)
{
    if (e->recycle)
        return pinned_take(e->device, bytes, p, cap);
    *cap = bytes;
    return (int)cudaMallocHost(p, bytes);
}

void ssae_pinned_free(ssa_engine *e, void *p, size_t cap)
{
    if (!p)
        return;
    if (e->recycle)
        pinned_return(e->device, p, cap);
    else
        cudaFreeHost(p);
}

#define dmalloc(pp, bytes) ssae_dalloc(e, (pp), (bytes))

int ssae_create(ssa_engine *e, int B, int N, int L, int kp, int k, cudaStream_t stream)
{
    memset(e, 0, sizeof(*e));
    if (B < 1 || N < 4 || L < 2 || L > N - 1 || kp < 1 || kp > SSA_MAX_KP || k < 1 || k > kp)
        return (int)cudaErrorInvalidValue;
    int logh = ssad_logh_for(N);
    if (logh > SSA_MAX_LOGH_ALL)
        return (int)cudaErrorInvalidValue;
    CK(cudaGetDevice(&e->device));
    CK(ssad_init_device());
    {
        const char *sc = getenv("SSA_SYNC_CHECK");
        e->sync_check = sc && sc[0] == '1';
    }
    e->B = B;
    e->N = N;
    e->L = L;
    e->K = N - L + 1;
    e->logh = logh;
    e->H = 1 << logh;
    e->kp = kp;
    e->k = k;
    e->ldL = round4(L);
    e->ldK = round4(e->K);
    e->ldN = round4(N);
    e->ldS = 2LL * (e->H + 1) + 2; /* floats; keeps every spectrum 16-byte aligned */
    e->ldS = round4(e->ldS);
    e->rows_L = gram_rows(L, B);
    e->rows_K = gram_rows(e->K, B);
    e->rows_N = imin(gram_rows(N, B), SSA_W_MAX_ROWS);
    e->nch_L = (L + e->rows_L - 1) / e->rows_L;
    e->nch_K = (e->K + e->rows_K - 1) / e->rows_K;
    e->nch_N = (N + e->rows_N - 1) / e->rows_N;
    e->nq = (L + SSA_ROWMUL_ROWS - 1) / SSA_ROWMUL_ROWS;
    if (stream)
    {
        e->st = stream;
    }
    else
    {
        e->recycle = g_recycle_on;
        if (e->recycle)
            CK(stream_take(e->device, &e->st));
        else
            CK(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
        e->own_stream = 1;
    }
    const size_t Bs = (size_t)B;
    const int nchmax = imax(e->nch_L, imax(e->nch_K, e->nch_N));
    const size_t np = (size_t)kp * (kp + 1) / 2;
    int r = 0;
    r |= dmalloc((void **)&e->x64, Bs * N * sizeof(double));
    r |= dmalloc((void **)&e->X, Bs * e->ldS * sizeof(float));
    r |= dmalloc((void **)&e->Y, Bs * e->ldL * kp * sizeof(float));
    r |= dmalloc((void **)&e->Z, Bs * e->ldK * kp * sizeof(float));
    r |= dmalloc((void **)&e->part, Bs * nchmax * np * sizeof(double));
    r |= dmalloc((void **)&e->qsum, Bs * e->nq * kp * sizeof(double));
    r |= dmalloc((void **)&e->Rinv, Bs * kp * kp * sizeof(double));
    r |= dmalloc((void **)&e->Zu, Bs * kp * k * sizeof(float));
    r |= dmalloc((void **)&e->Zv, Bs * kp * k * sizeof(float));
    r |= dmalloc((void **)&e->sigma, Bs * k * sizeof(double));
    r |= dmalloc((void **)&e->status, Bs * sizeof(int));
    r |= dmalloc((void **)&e->norm2, Bs * k * sizeof(double));
    r |= dmalloc((void **)&e->W, Bs * k * k * sizeof(double));
    if (r)
    {
        ssae_destroy(e);
        return (int)cudaErrorMemoryAllocation;
    }
    const size_t jbytes = (size_t)B * 8192 + (1 << 20);
    if (ssae_pinned(e, jbytes, (void **)&e->ja.h, &e->ja.hcap) != 0 ||
        ssae_dalloc(e, (void **)&e->ja.d, jbytes) != 0)
    {
        ssae_destroy(e);
        return (int)cudaErrorMemoryAllocation;
    }
    e->ja.cap = jbytes;
    CK(cudaMemsetAsync(e->status, 0, Bs * sizeof(int), e->st));
    return 0;
}

int ssae_create_light(ssa_engine *e, size_t arena_bytes, cudaStream_t stream)
{
    memset(e, 0, sizeof(*e));
    CK(cudaGetDevice(&e->device));
    CK(ssad_init_device());
    {
        const char *sc = getenv("SSA_SYNC_CHECK");
        e->sync_check = sc && sc[0] == '1';
    }
    if (stream)
    {
        e->st = stream;
    }
    else
    {
        /* recycled like a full engine: a growing job arena then frees in stream order and keeps
         * its old page-locked block for reuse, instead of synchronising the device */
        e->recycle = g_recycle_on;
        if (e->recycle)
            CK(stream_take(e->device, &e->st));
        else
            CK(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
        e->own_stream = 1;
    }
    return ssae_grow_arena(e, arena_bytes);
}

int ssae_grow_arena(ssa_engine *e, size_t bytes)
{
    if (bytes <= e->ja.cap)
        return 0;
    /* growing waits for this engine's stream (and, without recycling, frees that wait for the
     * whole device): at least double, so that a growing workload pays it a few times, not once
     * per batch */
    if (e->ja.cap > 0 && bytes < 2 * e->ja.cap)
        bytes = 2 * e->ja.cap;
    {
        const char *ev = getenv("SSA_SERVER_TRACE");
        if (ev && ev[0] == '1' && e->ja.cap > 0)
            fprintf(stderr, "ssa_engine: job arena grows %zu -> %zu bytes%s\n", e->ja.cap, bytes,
                    e->recycle ? "" : " (frees synchronise the device)");
    }
    if (e->st)
        CK(cudaStreamSynchronize(e->st));
    ssae_pinned_free(e, e->ja.h, e->ja.hcap);
    ssae_dfree(e, e->ja.d);
    e->ja.h = NULL;
    e->ja.d = NULL;
    e->ja.cap = 0;
    e->ja.hcap = 0;
    e->ja.used = 0;
    CK(ssae_pinned(e, bytes, (void **)&e->ja.h, &e->ja.hcap));
    CK(ssae_dalloc(e, (void **)&e->ja.d, bytes));
    e->ja.cap = bytes;
    return 0;
}

int ssae_set_profiling(ssa_engine *e, int on)
{
    if (on && !e->ev[0])
    {
        for (int i = 0; i < 2 * SSA_PROF_MAX; i++)
            if (cudaEventCreate(&e->ev[i]) != cudaSuccess)
                return -1;
    }
    e->prof = on;
    e->nev = 0;
    for (int k = 0; k < SSAK_NKINDS; k++)
    {
        e->prof_ms[k] = 0.0;
        e->prof_n[k] = 0;
    }
    return 0;
}

static const char *kind_name(int k)
{
    static const char *names[SSAK_NKINDS] = {"spectrum", "corr", "gram", "chol", "rowmul", "rr",
                                             "elem_recon", "wcorr_finish", "group_sum", "recon", "lrf",
                                             "wcorr_gram"};
    return (k >= 0 && k < SSAK_NKINDS) ? names[k] : "?";
}

void ssae_prof_begin(ssa_engine *e, int kind)
{
    e->cur_kind = kind;
    if (!e->prof || e->nev >= SSA_PROF_MAX)
        return;
    e->ev_kind[e->nev] = kind;
    cudaEventRecord(e->ev[2 * e->nev], e->st);
}

void ssae_prof_end(ssa_engine *e)
{
    if (e->sync_check)
    {
        cudaError_t err = cudaStreamSynchronize(e->st);
        if (err != cudaSuccess)
            fprintf(stderr, "ssa: stage %s failed: %s\n", kind_name(e->cur_kind), cudaGetErrorString(err));
    }
    if (!e->prof || e->nev >= SSA_PROF_MAX)
        return;
    cudaEventRecord(e->ev[2 * e->nev + 1], e->st);
    e->nev++;
}

int ssae_prof_collect(ssa_engine *e)
{
    if (!e->prof)
        return 0;
    if (cudaStreamSynchronize(e->st) != cudaSuccess)
        return -1;
    for (int i = 0; i < e->nev; i++)
    {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, e->ev[2 * i], e->ev[2 * i + 1]) != cudaSuccess)
            return -1;
        e->prof_ms[e->ev_kind[i]] += ms;
        e->prof_n[e->ev_kind[i]] += 1;
    }
    e->nev = 0;
    return 0;
}

void ssae_destroy(ssa_engine *e)
{
    if (!e)
        return;
    if (e->st)
        cudaStreamSynchronize(e->st);
    for (int i = 0; i < 2 * SSA_PROF_MAX; i++)
        if (e->ev[i])
            cudaEventDestroy(e->ev[i]);
    void *bufs[] = {e->x64, e->X, e->Y, e->Z, e->part, e->qsum, e->Rinv, e->Zu, e->Zv,
                    e->sigma, e->status, e->recon, e->norm2, e->W, e->Us, e->Vs, e->ja.d,
                    e->Ub, e->Vb, e->xpart, e->xC, e->sUs, e->sVs, e->sDinv, e->perm, e->sgn,
                    e->Ut, e->Vt, e->bsplit, e->Zs};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); i++)
        ssae_dfree(e, bufs[i]);
    ssae_pinned_free(e, e->ja.h, e->ja.hcap);
    if (e->own_stream && e->st)
    {
        if (e->recycle)
            stream_return(e->device, e->st);
        else
            cudaStreamDestroy(e->st);
    }
    memset(e, 0, sizeof(*e));
}

int ssae_ensure_recon(ssa_engine *e)
{
    if (e->recon)
        return 0;
    return dmalloc((void **)&e->recon, (size_t)e->B * e->k * e->ldN * sizeof(float));
}

int ssae_ensure_spectra(ssa_engine *e)
{
    size_t bytes = (size_t)e->B * e->k * e->ldS * sizeof(float);
    if (!e->Us)
        CK(dmalloc((void **)&e->Us, bytes));
    if (!e->Vs)
        CK(dmalloc((void **)&e->Vs, bytes));
    return 0;
}

/* Spectra of sigma_i u_i only (into Us), for the one-buffer elementary reconstruction. */
static int u_spectra(ssa_engine *e, int nb, int k)
{
    if (!e->Us)
        CK(dmalloc((void **)&e->Us, (size_t)e->B * e->k * e->ldS * sizeof(float)));
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)nb, sizeof(ssa_col_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int s = 0; s < nb; s++)
    {
        ssa_col_job *Ju = &jobs[s];
        Ju->in = e->Y + (size_t)s * e->ldL * e->kp;
        Ju->ld_in = e->ldL;
        Ju->n_in = e->L;
        Ju->scale = e->sigma + (size_t)s * e->k;
        Ju->spec = e->Us + (size_t)s * e->k * e->ldS;
        Ju->ld_spec = e->ldS;
        Ju->ncols = k;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_col_job) * nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_SPECTRUM);
    int rc_ = ssad_spectrum((const ssa_col_job *)d, nb, k, e->logh, e->st);
    ssae_prof_end(e);
    return rc_;
}

void ssae_reset_jobs(ssa_engine *e)
{
    cudaStreamSynchronize(e->st);
    if (e->prof)
        ssae_prof_collect(e);
    e->ja.used = 0;
}

void *ssae_push_jobs(ssa_engine *e, const void *jobs, size_t sz)
{
    size_t off = (e->ja.used + 15) & ~(size_t)15;
    if (off + sz > e->ja.cap)
        return NULL;
    memcpy(e->ja.h + off, jobs, sz);
    if (cudaMemcpyAsync(e->ja.d + off, e->ja.h + off, sz, cudaMemcpyHostToDevice, e->st) != cudaSuccess)
        return NULL;
    e->ja.used = off + sz;
    return e->ja.d + off;
}

int ssae_upload_jobs(ssa_engine *e)
{
    (void)e;
    return 0;
}

/* ------------------------------------------------------------------------------------------ */

int ssae_signal_spectrum(ssa_engine *e, const double *d_x, int nb)
{
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)nb, sizeof(ssa_col_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int s = 0; s < nb; s++)
    {
        ssa_col_job *J = &jobs[s];
        J->in64 = d_x + (size_t)s * e->N;
        J->ld_in = e->N;
        J->n_in = e->N;
        J->spec = e->X + (size_t)s * e->ldS;
        J->ld_spec = e->ldS;
        J->ncols = 1;
        J->N = e->N;
        J->L = e->L;
        J->K = e->K;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_col_job) * nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_SPECTRUM);
    int rc_ = ssad_spectrum((const ssa_col_job *)d, nb, 1, e->logh, e->st);
    ssae_prof_end(e);
    return rc_;
}

/* Correlation sweep: out = H in (fwd: in K rows -> out L rows) or H^T in (adjoint). */
static int sweep(ssa_engine *e, int nb, int ncols, int adjoint, const float *d_omega, long long omega_ld,
                 unsigned long long seed, int generate)
{
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)nb, sizeof(ssa_col_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int s = 0; s < nb; s++)
    {
        ssa_col_job *J = &jobs[s];
        float *Ys = e->Y + (size_t)s * e->ldL * e->kp;
        float *Zs = e->Z + (size_t)s * e->ldK * e->kp;
        if (!adjoint)
        {
            if (generate)
            {
                if (d_omega)
                {
                    J->in = d_omega + (size_t)s * omega_ld * ncols;
                    J->ld_in = omega_ld;
                }
                else
                {
                    J->in = NULL;
                    J->seed = seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(s + 1));
                }
            }
            else
            {
                J->in = Zs;
                J->ld_in = e->ldK;
            }
            J->n_in = e->K;
            J->out = Ys;
            J->ld_out = e->ldL;
            J->n_out = e->L;
        }
        else
        {
            J->in = Ys;
            J->ld_in = e->ldL;
            J->n_in = e->L;
            J->out = Zs;
            J->ld_out = e->ldK;
            J->n_out = e->K;
        }
        J->X = e->X + (size_t)s * e->ldS;
        J->ncols = ncols;
        J->N = e->N;
        J->L = e->L;
        J->K = e->K;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_col_job) * nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_CORR);
    int rc_ = ssad_corr((const ssa_col_job *)d, nb, ncols, e->logh, e->st);
    ssae_prof_end(e);
    return rc_;
}

int ssae_matvec(ssa_engine *e, int ncols, int adjoint)
{
    return sweep(e, 1, ncols, adjoint, NULL, 0, 0, 0);
}

/* Gram partials of the m x n blocks A_s (stride per series `sstride`, leading dim ld). */
static int gram_ps(ssa_engine *e, int nb, const float *A, size_t sstride, long long ld, int m, int n, int rows,
                   int weighted, size_t pstride);

static int gram(ssa_engine *e, int nb, const float *A, size_t sstride, long long ld, int m, int n, int rows,
                int weighted)
{
    const int nchmax = imax(e->nch_L, imax(e->nch_K, e->nch_N));
    return gram_ps(e, nb, A, sstride, ld, m, n, rows, weighted, (size_t)nchmax * e->kp * (e->kp + 1) / 2);
}

/* Gram partials with series s's partials at e->part + s * pstride. */
static int gram_ps(ssa_engine *e, int nb, const float *A, size_t sstride, long long ld, int m, int n, int rows,
                   int weighted, size_t pstride)
{
    ssa_gram_job *jobs = (ssa_gram_job *)calloc((size_t)nb, sizeof(ssa_gram_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    const int nch = (m + rows - 1) / rows;
    for (int s = 0; s < nb; s++)
    {
        ssa_gram_job *J = &jobs[s];
        J->A = A + (size_t)s * sstride;
        J->part = e->part + (size_t)s * pstride;
        J->ld = ld;
        J->m = m;
        J->n = n;
        J->rows_per_cta = rows;
        J->weighted = weighted;
        J->N = e->N;
        J->L = e->L;
        J->K = e->K;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_gram_job) * nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, weighted ? SSAK_WGRAM : SSAK_GRAM);
    int rc_ = ssad_gram((const ssa_gram_job *)d, nb, nch, weighted, e->st);
    ssae_prof_end(e);
    return rc_;
}

static int chol(ssa_engine *e, int nb, int nch, int n)
{
    ssa_chol_job *jobs = (ssa_chol_job *)calloc((size_t)nb, sizeof(ssa_chol_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    const int nchmax = imax(e->nch_L, imax(e->nch_K, e->nch_N));
    const size_t np = (size_t)e->kp * (e->kp + 1) / 2;
    for (int s = 0; s < nb; s++)
    {
        ssa_chol_job *J = &jobs[s];
        J->part = e->part + (size_t)s * nchmax * np;
        J->Rinv = e->Rinv + (size_t)s * e->kp * e->kp;
        J->status = e->status + s;
        J->nchunks = nch;
        J->n = n;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_chol_job) * nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_CHOL);
    int rc_ = ssad_chol((const ssa_chol_job *)d, nb, e->st);
    ssae_prof_end(e);
    return rc_;
}

/* C_s = A_s * M_s for all series (M_s small, n x p, ld ldb, per-series stride mstride; FP32 Mm,
 * or FP64 Mm64 when that is given). */
static int rowmul(ssa_engine *e, int nb, const float *A, size_t astride, long long lda, int m, int n,
                  const float *Mm, size_t mstride, int ldb, int p, float *C, size_t cstride, long long ldc,
                  double *colsum, const double *Mm64)
{
    ssa_rowmul_job *jobs = (ssa_rowmul_job *)calloc((size_t)nb, sizeof(ssa_rowmul_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    const int nqb = (m + SSA_ROWMUL_ROWS - 1) / SSA_ROWMUL_ROWS;
    for (int s = 0; s < nb; s++)
    {
        ssa_rowmul_job *J = &jobs[s];
        J->A = A + (size_t)s * astride;
        J->Bm = Mm64 ? NULL : Mm + (size_t)s * mstride;
        J->Bm64 = Mm64 ? Mm64 + (size_t)s * mstride : NULL;
        J->C = C + (size_t)s * cstride;
        J->colsum = colsum ? colsum + (size_t)s * nqb * p : NULL;
        J->lda = lda;
        J->ldc = ldc;
        J->m = m;
        J->n = n;
        J->p = p;
        J->ldb = ldb;
    }
    const int tc = !e->rowmul_simt && ssad_rowmul_tc_on();
    if (tc && (size_t)nb > e->bsplit_cap)
    {
        ssae_dfree(e, e->bsplit);
        e->bsplit = NULL;
        e->bsplit_cap = 0;
        if (ssae_dalloc(e, (void **)&e->bsplit, sizeof(float) * SSA_ROWMUL_BSPLIT_FLOATS * (size_t)nb) != 0)
        {
            free(jobs);
            return (int)cudaErrorMemoryAllocation;
        }
        e->bsplit_cap = (size_t)nb;
    }
    if (tc)
        for (int s = 0; s < nb; s++)
            jobs[s].Bsplit = e->bsplit + (size_t)s * SSA_ROWMUL_BSPLIT_FLOATS;
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_rowmul_job) * nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_ROWMUL);
    int rc_ = tc ? ssad_rowmul_tc((const ssa_rowmul_job *)d, nb, m, n, e->st)
                 : ssad_rowmul((const ssa_rowmul_job *)d, nb, m, n, e->st);
    ssae_prof_end(e);
    return rc_;
}

/* One CholQR pass on the m x n blocks A_s in place. */
static int cholqr_pass(ssa_engine *e, int nb, float *A, size_t sstride, long long ld, int m, int n, int rows,
                       double *colsum)
{
    const int nch = (m + rows - 1) / rows;
    CK(gram(e, nb, A, sstride, ld, m, n, rows, 0));
    CK(chol(e, nb, nch, n));
    return rowmul(e, nb, A, sstride, ld, m, n, NULL, (size_t)e->kp * e->kp, n, n, A, sstride, ld, colsum, e->Rinv);
}

int ssae_decompose(ssa_engine *e, int nb, int kp, int k, int q, const float *d_omega, long long omega_ld,
                   unsigned long long seed)
{
    if (nb < 1 || nb > e->B || kp < 1 || kp > e->kp || k < 1 || k > imin(kp, e->k))
        return (int)cudaErrorInvalidValue;
    const size_t sY = (size_t)e->ldL * e->kp, sZ = (size_t)e->ldK * e->kp;
    const int L = e->L, K = e->K;
    CK(cudaMemsetAsync(e->status, 0, sizeof(int) * nb, e->st));
    /* Y = H Omega */
    CK(sweep(e, nb, kp, 0, d_omega, omega_ld, seed, 1));
    for (int it = 0; it < q; it++)
    {
        /* Intermediate bases need to be well conditioned, not orthonormal to rounding: one
         * CholQR pass (FP64 Gram, so the loss of orthogonality is ~u32 cond(Y)).
         * Q = orth(Y), Z = H^T Q, Z = orth(Z), Y = H Z */
        CK(cholqr_pass(e, nb, e->Y, sY, e->ldL, L, kp, e->rows_L, NULL));
        CK(sweep(e, nb, kp, 1, NULL, 0, 0, 0));
        CK(cholqr_pass(e, nb, e->Z, sZ, e->ldK, K, kp, e->rows_K, NULL));
        CK(sweep(e, nb, kp, 0, NULL, 0, 0, 0));
    }
    /* final Q = CholQR2(Y) with the column sums of Q for the sign rule */
    CK(cholqr_pass(e, nb, e->Y, sY, e->ldL, L, kp, e->rows_L, NULL));
    CK(cholqr_pass(e, nb, e->Y, sY, e->ldL, L, kp, e->rows_L, e->qsum));
    /* B = H^T Q */
    CK(sweep(e, nb, kp, 1, NULL, 0, 0, 0));
    /* Rayleigh-Ritz on B^T B */
    CK(gram(e, nb, e->Z, sZ, e->ldK, K, kp, e->rows_K, 0));
    {
        ssa_rr_job *jobs = (ssa_rr_job *)calloc((size_t)nb, sizeof(ssa_rr_job));
        if (!jobs)
            return (int)cudaErrorMemoryAllocation;
        const int nchmax = imax(e->nch_L, imax(e->nch_K, e->nch_N));
        const size_t np = (size_t)e->kp * (e->kp + 1) / 2;
        const int nqb = (L + SSA_ROWMUL_ROWS - 1) / SSA_ROWMUL_ROWS;
        for (int s = 0; s < nb; s++)
        {
            ssa_rr_job *J = &jobs[s];
            J->part = e->part + (size_t)s * nchmax * np;
            J->qsum = e->qsum + (size_t)s * nqb * kp;
            J->sigma = e->sigma + (size_t)s * e->k;
            J->Zu = e->Zu + (size_t)s * e->kp * e->k;
            J->Zv = e->Zv + (size_t)s * e->kp * e->k;
            J->status = e->status + s;
            J->nchunks = (K + e->rows_K - 1) / e->rows_K;
            J->nchunks_q = nqb;
            J->kp = kp;
            J->k = k;
        }
        void *d = ssae_push_jobs(e, jobs, sizeof(ssa_rr_job) * nb);
        free(jobs);
        if (!d)
            return (int)cudaErrorMemoryAllocation;
        ssae_prof_begin(e, SSAK_RR);
        int rc_ = ssad_rr((const ssa_rr_job *)d, nb, e->st);
        ssae_prof_end(e);
        CK(rc_);
    }
    /* U = Q Zu (in place over Y), V = B Zv (in place over Z) */
    CK(rowmul(e, nb, e->Y, sY, e->ldL, L, kp, e->Zu, (size_t)e->kp * e->k, kp, k, e->Y, sY, e->ldL, NULL, NULL));
    CK(rowmul(e, nb, e->Z, sZ, e->ldK, K, kp, e->Zv, (size_t)e->kp * e->k, kp, k, e->Z, sZ, e->ldK, NULL, NULL));
    return 0;
}

int ssae_elem_recon(ssa_engine *e, int nb, int k)
{
    CK(ssae_ensure_recon(e));
    const int one_buffer = e->logh > SSA_ELEM2_MAX_LOGH;
    if (one_buffer)
        CK(u_spectra(e, nb, k));
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)nb, sizeof(ssa_col_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int s = 0; s < nb; s++)
    {
        ssa_col_job *J = &jobs[s];
        J->in = e->Y + (size_t)s * e->ldL * e->kp;
        J->ld_in = e->ldL;
        J->n_in = e->L;
        J->in2 = e->Z + (size_t)s * e->ldK * e->kp;
        J->ld_in2 = e->ldK;
        J->n_in2 = e->K;
        J->scale = e->sigma + (size_t)s * e->k;
        J->out = e->recon + (size_t)s * e->k * e->ldN;
        J->ld_out = e->ldN;
        J->norm2 = e->norm2 + (size_t)s * e->k;
        J->ncols = k;
        J->N = e->N;
        J->L = e->L;
        J->K = e->K;
        if (one_buffer)
        {
            J->spec = e->Us + (size_t)s * e->k * e->ldS;
            J->ld_spec = e->ldS;
        }
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_col_job) * nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_ELEM);
    int rc_ = one_buffer ? ssad_elem_recon1((const ssa_col_job *)d, nb, k, e->logh, e->st)
                         : ssad_elem_recon((const ssa_col_job *)d, nb, k, e->logh, e->st);
    ssae_prof_end(e);
    return rc_;
}

/* W-correlation Gram on the tensor cores: chunks of at least SSA_TC_MIN_ROWS time steps. */
static int wgram_tc(ssa_engine *e, int nb, int k, int rows)
{
    const int nchmax = imax(e->nch_L, imax(e->nch_K, e->nch_N));
    const size_t np = (size_t)e->kp * (e->kp + 1) / 2;
    ssa_wgram_job *jobs = (ssa_wgram_job *)calloc((size_t)nb, sizeof(ssa_wgram_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int s = 0; s < nb; s++)
    {
        ssa_gram_job *J = &jobs[s].g;
        jobs[s].status = e->status + s;
        J->A = e->recon + (size_t)s * e->k * e->ldN;
        J->part = e->part + (size_t)s * nchmax * np;
        J->ld = e->ldN;
        J->m = e->N;
        J->n = k;
        J->rows_per_cta = rows;
        J->weighted = 1;
        J->N = e->N;
        J->L = e->L;
        J->K = e->K;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_wgram_job) * nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_WGRAM);
    int rc_ = ssad_gram_tc((const ssa_wgram_job *)d, nb, (e->N + rows - 1) / rows, e->st);
    ssae_prof_end(e);
    return rc_;
}

int ssae_wcorr(ssa_engine *e, int nb, int k)
{
    /* weighted Gram of the elementary reconstructions: G_ij = sum_t w_t x~_i[t] x~_j[t], on the
     * tensor cores (split TF32) or with FP64 accumulation on the CUDA cores */
    const int tc = ssad_wcorr_tc();
    const int rows_tc = imax(e->rows_N, SSA_TC_MIN_ROWS);
    const int nch_w = tc ? (e->N + rows_tc - 1) / rows_tc : e->nch_N;
    if (tc)
        CK(wgram_tc(e, nb, k, rows_tc));
    else
        CK(gram(e, nb, e->recon, (size_t)e->k * e->ldN, e->ldN, e->N, k, e->rows_N, 1));
    ssa_wfin_job *jobs = (ssa_wfin_job *)calloc((size_t)nb, sizeof(ssa_wfin_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    const int nchmax = imax(e->nch_L, imax(e->nch_K, e->nch_N));
    const size_t np = (size_t)e->kp * (e->kp + 1) / 2;
    for (int s = 0; s < nb; s++)
    {
        jobs[s].part = e->part + (size_t)s * nchmax * np;
        jobs[s].W = e->W + (size_t)s * e->k * e->k;
        jobs[s].nchunks = nch_w;
        jobs[s].k = k;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_wfin_job) * nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_WFIN);
    int rc_ = ssad_wfin((const ssa_wfin_job *)d, nb, e->st);
    ssae_prof_end(e);
    return rc_;
}

int ssae_spectra(ssa_engine *e, int nb, int k)
{
    CK(ssae_ensure_spectra(e));
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)nb * 2, sizeof(ssa_col_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int s = 0; s < nb; s++)
    {
        ssa_col_job *Ju = &jobs[2 * s], *Jv = &jobs[2 * s + 1];
        Ju->in = e->Y + (size_t)s * e->ldL * e->kp;
        Ju->ld_in = e->ldL;
        Ju->n_in = e->L;
        Ju->scale = e->sigma + (size_t)s * e->k;
        Ju->spec = e->Us + (size_t)s * e->k * e->ldS;
        Ju->ld_spec = e->ldS;
        Ju->ncols = k;
        Jv->in = e->Z + (size_t)s * e->ldK * e->kp;
        Jv->ld_in = e->ldK;
        Jv->n_in = e->K;
        Jv->spec = e->Vs + (size_t)s * e->k * e->ldS;
        Jv->ld_spec = e->ldS;
        Jv->ncols = k;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_col_job) * nb * 2);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_SPECTRUM);
    int rc_ = ssad_spectrum((const ssa_col_job *)d, 2 * nb, k, e->logh, e->st);
    ssae_prof_end(e);
    return rc_;
}

int ssae_recon_group(ssa_engine *e, int s, int k, const int *d_group, int n_group, double *d_out)
{
    ssa_recon_job J;
    memset(&J, 0, sizeof(J));
    J.Us = e->Us + (size_t)s * e->k * e->ldS;
    J.Vs = e->Vs + (size_t)s * e->k * e->ldS;
    J.U = e->Y + (size_t)s * e->ldL * e->kp;
    J.V = e->Z + (size_t)s * e->ldK * e->kp;
    J.ldU = e->ldL;
    J.ldV = e->ldK;
    J.sigma = e->sigma + (size_t)s * e->k;
    J.group = d_group;
    J.out64 = d_out;
    J.ld_spec = e->ldS;
    J.n_group = n_group;
    J.k = k;
    J.N = e->N;
    J.L = e->L;
    J.K = e->K;
    void *d = ssae_push_jobs(e, &J, sizeof(J));
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_RECON);
    int rc_ = ssad_recon((const ssa_recon_job *)d, 1, e->logh, e->st);
    ssae_prof_end(e);
    return rc_;
}

/* ------------------------------------------------------------------------------------------ */
/* Block power iteration                                                                       */
/* ------------------------------------------------------------------------------------------ */

int ssae_ensure_block(ssa_engine *e, int bcap)
{
    if (e->Ub && e->bcap >= bcap)
        return 0;
    void *old[] = {e->Ub, e->Vb, e->xpart, e->xC, e->sUs, e->sVs, e->sDinv, e->perm, e->sgn, e->Ut, e->Vt};
    cudaStreamSynchronize(e->st);
    for (size_t i = 0; i < sizeof(old) / sizeof(old[0]); i++)
        ssae_dfree(e, old[i]);
    const size_t Bs = (size_t)e->B;
    const int nchx = imax(e->nch_L, e->nch_K);
    int r = 0;
    r |= dmalloc((void **)&e->Ub, Bs * e->ldL * 2 * bcap * sizeof(float));
    r |= dmalloc((void **)&e->Vb, Bs * e->ldK * bcap * sizeof(float));
    r |= dmalloc((void **)&e->xpart, Bs * nchx * SSA_MAX_KP * SSA_MAX_KP * sizeof(double));
    r |= dmalloc((void **)&e->xC, Bs * SSA_MAX_KP * SSA_MAX_KP * sizeof(float));
    r |= dmalloc((void **)&e->sUs, Bs * SSA_MAX_KP * SSA_MAX_KP * sizeof(float));
    r |= dmalloc((void **)&e->sVs, Bs * SSA_MAX_KP * SSA_MAX_KP * sizeof(float));
    r |= dmalloc((void **)&e->sDinv, Bs * SSA_MAX_KP * SSA_MAX_KP * sizeof(float));
    r |= dmalloc((void **)&e->perm, Bs * SSA_MAX_KP * sizeof(int));
    r |= dmalloc((void **)&e->sgn, Bs * SSA_MAX_KP * sizeof(float));
    r |= dmalloc((void **)&e->Ut, Bs * e->ldL * e->kp * sizeof(float));
    r |= dmalloc((void **)&e->Vt, Bs * e->ldK * e->kp * sizeof(float));
    e->bcap = r ? 0 : bcap;
    return r ? (int)cudaErrorMemoryAllocation : 0;
}

/* out_s = H in_s (adjoint = 0: in K rows, out L rows) or H^T in_s, ncols columns. */
static int corr_io(ssa_engine *e, int nb, int ncols, int adjoint, const float *in, size_t in_stride, long long ld_in,
                   float *out, size_t out_stride, long long ld_out)
{
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)nb, sizeof(ssa_col_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int s = 0; s < nb; s++)
    {
        ssa_col_job *J = &jobs[s];
        J->in = in + (size_t)s * in_stride;
        J->ld_in = ld_in;
        J->n_in = adjoint ? e->L : e->K;
        J->out = out + (size_t)s * out_stride;
        J->ld_out = ld_out;
        J->n_out = adjoint ? e->K : e->L;
        J->X = e->X + (size_t)s * e->ldS;
        J->ncols = ncols;
        J->N = e->N;
        J->L = e->L;
        J->K = e->K;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_col_job) * nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_CORR);
    int rc_ = ssad_corr((const ssa_col_job *)d, nb, ncols, e->logh, e->st);
    ssae_prof_end(e);
    return rc_;
}

/* X_s -= Q_s (Q_s^T X_s): Q_s m x nq (ldq), X_s m x nx (ldx); FP64-accumulated cross products. */
static int deflate(ssa_engine *e, int nb, float *Xm, size_t xs, long long ldx, int nx, const float *Q, size_t qs,
                   long long ldq, int nq, int m, int rows)
{
    const int nch = (m + rows - 1) / rows;
    const int nchx = imax(e->nch_L, e->nch_K);
    ssa_xgram_job *xg = (ssa_xgram_job *)calloc((size_t)nb, sizeof(ssa_xgram_job));
    ssa_xreduce_job *xr = (ssa_xreduce_job *)calloc((size_t)nb, sizeof(ssa_xreduce_job));
    if (!xg || !xr)
    {
        free(xg);
        free(xr);
        return (int)cudaErrorMemoryAllocation;
    }
    for (int s = 0; s < nb; s++)
    {
        xg[s].A = Q + (size_t)s * qs;
        xg[s].B = Xm + (size_t)s * xs;
        xg[s].part = e->xpart + (size_t)s * nchx * SSA_MAX_KP * SSA_MAX_KP;
        xg[s].lda = ldq;
        xg[s].ldb = ldx;
        xg[s].m = m;
        xg[s].na = nq;
        xg[s].nb = nx;
        xg[s].rows_per_cta = rows;
        xr[s].part = xg[s].part;
        xr[s].out = e->xC + (size_t)s * SSA_MAX_KP * SSA_MAX_KP;
        xr[s].nchunks = nch;
        xr[s].na = nq;
        xr[s].nb = nx;
    }
    void *dg = ssae_push_jobs(e, xg, sizeof(ssa_xgram_job) * nb);
    void *dr = ssae_push_jobs(e, xr, sizeof(ssa_xreduce_job) * nb);
    free(xg);
    free(xr);
    if (!dg || !dr)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_GRAM);
    int rc = ssad_xgram((const ssa_xgram_job *)dg, nb, nch, e->st);
    ssae_prof_end(e);
    CK(rc);
    ssae_prof_begin(e, SSAK_GRAM);
    rc = ssad_xreduce((const ssa_xreduce_job *)dr, nb, e->st);
    ssae_prof_end(e);
    CK(rc);
    /* X = X - Q C */
    ssa_rowmul_job *rj = (ssa_rowmul_job *)calloc((size_t)nb, sizeof(ssa_rowmul_job));
    if (!rj)
        return (int)cudaErrorMemoryAllocation;
    for (int s = 0; s < nb; s++)
    {
        ssa_rowmul_job *J = &rj[s];
        J->A = Q + (size_t)s * qs;
        J->Bm = e->xC + (size_t)s * SSA_MAX_KP * SSA_MAX_KP;
        J->C = Xm + (size_t)s * xs;
        J->sub = Xm + (size_t)s * xs;
        J->lda = ldq;
        J->ldc = ldx;
        J->ldsub = ldx;
        J->m = m;
        J->n = nq;
        J->p = nx;
        J->ldb = nq;
    }
    void *d = ssae_push_jobs(e, rj, sizeof(ssa_rowmul_job) * nb);
    free(rj);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_ROWMUL);
    rc = ssad_rowmul((const ssa_rowmul_job *)d, nb, m, nq, e->st);
    ssae_prof_end(e);
    return rc;
}

/* Block power iteration for components [comp0, k); components [0, comp0) are already in Y, Z
 * and sigma (deflated against, re-sorted with the new ones, their signs kept). */
static int block_power_run(ssa_engine *e, int nb, int k, int comp0, int bsize, int max_iter, const float *d_V0,
                           long long v0_ld, unsigned long long seed);

/* Block power keeps its row products on the CUDA cores: it orthonormalises only every few
 * iterations, and amplifies the rounding of the products in between by (sigma_1 / sigma_k)^(2j). */
static int block_power(ssa_engine *e, int nb, int k, int comp0, int bsize, int max_iter, const float *d_V0,
                       long long v0_ld, unsigned long long seed)
{
    const int saved = e->rowmul_simt;
    e->rowmul_simt = 1;
    const int rc = block_power_run(e, nb, k, comp0, bsize, max_iter, d_V0, v0_ld, seed);
    e->rowmul_simt = saved;
    return rc;
}

static int block_power_run(ssa_engine *e, int nb, int k, int comp0, int bsize, int max_iter, const float *d_V0,
                           long long v0_ld, unsigned long long seed)
{
    const int L = e->L, K = e->K;
    if (nb < 1 || nb > e->B || k < 1 || bsize < 1 || max_iter < 0 || comp0 < 0)
        return (int)cudaErrorInvalidValue;
    k = imin(k, imin(L, K));
    if (comp0 >= k)
        return (int)cudaErrorInvalidValue;
    const int b = imin(bsize, k);
    if (k > e->kp || k > e->k || b > SSA_MAX_KP)
        return (int)cudaErrorInvalidValue;
    CK(ssae_ensure_block(e, b));
    CK(cudaMemsetAsync(e->status, 0, sizeof(int) * nb, e->st));
    const size_t sY = (size_t)e->ldL * e->kp, sZ = (size_t)e->ldK * e->kp;
    const size_t sUb = (size_t)e->ldL * 2 * e->bcap, sVb = (size_t)e->ldK * e->bcap;
    float *Ub = e->Ub, *Ub2 = e->Ub + (size_t)e->ldL * e->bcap, *Vb = e->Vb;
    const size_t s64 = (size_t)SSA_MAX_KP * SSA_MAX_KP;
    int comp = comp0;
    while (comp < k)
    {
        const int cb = imin(b, k - comp);
        /* start block */
        for (int s = 0; s < nb; s++)
        {
            if (d_V0)
                CK(cudaMemcpy2DAsync(Vb + (size_t)s * sVb, sizeof(float) * e->ldK,
                                     d_V0 + (size_t)s * v0_ld * k + (size_t)comp * v0_ld, sizeof(float) * v0_ld,
                                     sizeof(float) * K, cb, cudaMemcpyDeviceToDevice, e->st));
            else
                CK(ssad_gaussian(Vb + (size_t)s * sVb, e->ldK, K, cb, comp,
                                 seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(s + 1)), e->st));
        }
        if (comp > 0)
            CK(deflate(e, nb, Vb, sVb, e->ldK, cb, e->Z, sZ, e->ldK, comp, K, e->rows_K));
        CK(cholqr_pass(e, nb, Vb, sVb, e->ldK, K, cb, e->rows_K, NULL));
        CK(cholqr_pass(e, nb, Vb, sVb, e->ldK, K, cb, e->rows_K, NULL));
        for (int it = 0; it < max_iter; it++)
        {
            const int last = it == max_iter - 1;
            /* FP32 iterates are re-orthonormalised every half-step (the reference: every fifth),
             * which keeps the subspaces identical and avoids FP32 overflow. */
            CK(corr_io(e, nb, cb, 0, Vb, sVb, e->ldK, Ub, sUb, e->ldL));
            if (comp > 0)
                CK(deflate(e, nb, Ub, sUb, e->ldL, cb, e->Y, sY, e->ldL, comp, L, e->rows_L));
            CK(cholqr_pass(e, nb, Ub, sUb, e->ldL, L, cb, e->rows_L, NULL));
            if (last)
                CK(cholqr_pass(e, nb, Ub, sUb, e->ldL, L, cb, e->rows_L, NULL));
            CK(corr_io(e, nb, cb, 1, Ub, sUb, e->ldL, Vb, sVb, e->ldK));
            if (comp > 0)
                CK(deflate(e, nb, Vb, sVb, e->ldK, cb, e->Z, sZ, e->ldK, comp, K, e->rows_K));
            CK(cholqr_pass(e, nb, Vb, sVb, e->ldK, K, cb, e->rows_K, NULL));
            if (last)
                CK(cholqr_pass(e, nb, Vb, sVb, e->ldK, K, cb, e->rows_K, NULL));
        }
        /* U_block2 = H V_block (deflated); M = U_block^T U_block2 = Us S Vs^T */
        CK(corr_io(e, nb, cb, 0, Vb, sVb, e->ldK, Ub2, sUb, e->ldL));
        if (comp > 0)
            CK(deflate(e, nb, Ub2, sUb, e->ldL, cb, e->Y, sY, e->ldL, comp, L, e->rows_L));
        {
            const int nch = (L + e->rows_L - 1) / e->rows_L;
            const int nchx = imax(e->nch_L, e->nch_K);
            ssa_xgram_job *xg = (ssa_xgram_job *)calloc((size_t)nb, sizeof(ssa_xgram_job));
            ssa_svd_job *sv = (ssa_svd_job *)calloc((size_t)nb, sizeof(ssa_svd_job));
            if (!xg || !sv)
            {
                free(xg);
                free(sv);
                return (int)cudaErrorMemoryAllocation;
            }
            for (int s = 0; s < nb; s++)
            {
                xg[s].A = Ub + (size_t)s * sUb;
                xg[s].B = Ub2 + (size_t)s * sUb;
                xg[s].part = e->xpart + (size_t)s * nchx * s64;
                xg[s].lda = e->ldL;
                xg[s].ldb = e->ldL;
                xg[s].m = L;
                xg[s].na = cb;
                xg[s].nb = cb;
                xg[s].rows_per_cta = e->rows_L;
                sv[s].part = xg[s].part;
                sv[s].sigma = e->sigma + (size_t)s * e->k + comp;
                sv[s].Us = e->sUs + (size_t)s * s64;
                sv[s].Vs = e->sVs + (size_t)s * s64;
                sv[s].Dinv = e->sDinv + (size_t)s * s64;
                sv[s].status = e->status + s;
                sv[s].nchunks = nch;
                sv[s].n = cb;
            }
            void *dg = ssae_push_jobs(e, xg, sizeof(ssa_xgram_job) * nb);
            void *ds = ssae_push_jobs(e, sv, sizeof(ssa_svd_job) * nb);
            free(xg);
            free(sv);
            if (!dg || !ds)
                return (int)cudaErrorMemoryAllocation;
            ssae_prof_begin(e, SSAK_GRAM);
            int rc = ssad_xgram((const ssa_xgram_job *)dg, nb, nch, e->st);
            ssae_prof_end(e);
            CK(rc);
            ssae_prof_begin(e, SSAK_RR);
            rc = ssad_svdsmall((const ssa_svd_job *)ds, nb, e->st);
            ssae_prof_end(e);
            CK(rc);
        }
        /* U[:, comp:comp+cb] = U_block Us */
        CK(rowmul(e, nb, Ub, sUb, e->ldL, L, cb, e->sUs, s64, cb, cb, e->Y + (size_t)comp * e->ldL, sY, e->ldL,
                  NULL, NULL));
        /* V_block = H^T U[:, comp:comp+cb] (deflated); V[:, comp:comp+cb] = V_block Sigma^{-1} */
        CK(corr_io(e, nb, cb, 1, e->Y + (size_t)comp * e->ldL, sY, e->ldL, Vb, sVb, e->ldK));
        if (comp > 0)
            CK(deflate(e, nb, Vb, sVb, e->ldK, cb, e->Z, sZ, e->ldK, comp, K, e->rows_K));
        CK(rowmul(e, nb, Vb, sVb, e->ldK, K, cb, e->sDinv, s64, cb, cb, e->Z + (size_t)comp * e->ldK, sZ, e->ldK,
                  NULL, NULL));
        comp += cb;
    }
    /* exchange sort by sigma and sign rule (MKL/ssa_opt.h:1896-1919) */
    {
        ssa_sortsign_job *ss = (ssa_sortsign_job *)calloc((size_t)nb, sizeof(ssa_sortsign_job));
        ssa_permcols_job *pc = (ssa_permcols_job *)calloc((size_t)nb * 4, sizeof(ssa_permcols_job));
        if (!ss || !pc)
        {
            free(ss);
            free(pc);
            return (int)cudaErrorMemoryAllocation;
        }
        for (int s = 0; s < nb; s++)
        {
            ss[s].U = e->Y + (size_t)s * sY;
            ss[s].sigma = e->sigma + (size_t)s * e->k;
            ss[s].perm = e->perm + (size_t)s * SSA_MAX_KP;
            ss[s].sign = e->sgn + (size_t)s * SSA_MAX_KP;
            ss[s].ldU = e->ldL;
            ss[s].L = L;
            ss[s].k = k;
            ss[s].sign_from = comp0;
            /* Y -> Ut and Z -> Vt permuted, then copied back unpermuted-identity */
            ssa_permcols_job *a = &pc[4 * s];
            a[0].src = e->Y + (size_t)s * sY;
            a[0].dst = e->Ut + (size_t)s * sY;
            a[0].lds = a[0].ldd = e->ldL;
            a[0].m = L;
            a[1].src = e->Z + (size_t)s * sZ;
            a[1].dst = e->Vt + (size_t)s * sZ;
            a[1].lds = a[1].ldd = e->ldK;
            a[1].m = K;
            for (int t = 0; t < 2; t++)
            {
                a[t].perm = ss[s].perm;
                a[t].sign = ss[s].sign;
                a[t].k = k;
            }
        }
        void *dss = ssae_push_jobs(e, ss, sizeof(ssa_sortsign_job) * nb);
        free(ss);
        if (!dss)
        {
            free(pc);
            return (int)cudaErrorMemoryAllocation;
        }
        ssae_prof_begin(e, SSAK_RR);
        int rc = ssad_sortsign((const ssa_sortsign_job *)dss, nb, e->st);
        ssae_prof_end(e);
        if (rc)
        {
            free(pc);
            return rc;
        }
        /* permute U and V into the staging buffers, then copy them back */
        ssa_permcols_job *pu = (ssa_permcols_job *)calloc((size_t)nb, sizeof(ssa_permcols_job));
        ssa_permcols_job *pv = (ssa_permcols_job *)calloc((size_t)nb, sizeof(ssa_permcols_job));
        if (!pu || !pv)
        {
            free(pc);
            free(pu);
            free(pv);
            return (int)cudaErrorMemoryAllocation;
        }
        for (int s = 0; s < nb; s++)
        {
            pu[s] = pc[4 * s];
            pv[s] = pc[4 * s + 1];
        }
        free(pc);
        void *dpu = ssae_push_jobs(e, pu, sizeof(ssa_permcols_job) * nb);
        void *dpv = ssae_push_jobs(e, pv, sizeof(ssa_permcols_job) * nb);
        free(pu);
        free(pv);
        if (!dpu || !dpv)
            return (int)cudaErrorMemoryAllocation;
        CK(ssad_permcols((const ssa_permcols_job *)dpu, nb, L, e->st));
        CK(ssad_permcols((const ssa_permcols_job *)dpv, nb, K, e->st));
        for (int s = 0; s < nb; s++)
        {
            CK(cudaMemcpy2DAsync(e->Y + (size_t)s * sY, sizeof(float) * e->ldL, e->Ut + (size_t)s * sY,
                                 sizeof(float) * e->ldL, sizeof(float) * L, k, cudaMemcpyDeviceToDevice, e->st));
            CK(cudaMemcpy2DAsync(e->Z + (size_t)s * sZ, sizeof(float) * e->ldK, e->Vt + (size_t)s * sZ,
                                 sizeof(float) * e->ldK, sizeof(float) * K, k, cudaMemcpyDeviceToDevice, e->st));
        }
    }
    return 0;
}

int ssae_decompose_block(ssa_engine *e, int nb, int k, int bsize, int max_iter, const float *d_V0, long long v0_ld,
                         unsigned long long seed)
{
    return block_power(e, nb, k, 0, bsize, max_iter, d_V0, v0_ld, seed);
}

int ssae_extend(ssa_engine *e, int k_old, int k_new, int max_iter, unsigned long long seed)
{
    return block_power(e, 1, k_new, k_old, 1, max_iter, NULL, 0, seed);
}

/* ------------------------------------------------------------------------------------------ */
/* MSSA: M channels of one instance are the engine's series; the stacked (M L) x K operator    */
/* (reference MKL/ssa_opt.h:4069-4114) is applied channel by channel.                          */
/* ------------------------------------------------------------------------------------------ */

/* One CholQR pass on the stacked block [Y_0; ...; Y_{M-1}] (each L x n): Gram = sum of the
 * channel Grams, one Cholesky, the same R applied to every channel. */
static int mssa_cholqr(ssa_engine *e, int M, int n, double *colsum)
{
    const size_t sY = (size_t)e->ldL * e->kp;
    const int nch = (e->L + e->rows_L - 1) / e->rows_L;
    const size_t np = (size_t)n * (n + 1) / 2;
    CK(gram_ps(e, M, e->Y, sY, e->ldL, e->L, n, e->rows_L, 0, (size_t)nch * np));
    ssa_chol_job J;
    memset(&J, 0, sizeof(J));
    J.part = e->part;
    J.Rinv = e->Rinv;
    J.status = e->status;
    J.nchunks = M * nch;
    J.n = n;
    void *d = ssae_push_jobs(e, &J, sizeof(J));
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_CHOL);
    int rc = ssad_chol((const ssa_chol_job *)d, 1, e->st);
    ssae_prof_end(e);
    CK(rc);
    return rowmul(e, M, e->Y, sY, e->ldL, e->L, n, NULL, 0, n, n, e->Y, sY, e->ldL, colsum, e->Rinv);
}

/* Z_0 = sum_m H_m^T Y_m (per-channel adjoints into Z_m, then a fixed-order channel sum). */
static int mssa_adjoint(ssa_engine *e, int M, int n)
{
    const size_t sY = (size_t)e->ldL * e->kp, sZ = (size_t)e->ldK * e->kp;
    CK(corr_io(e, M, n, 1, e->Y, sY, e->ldL, e->Z, sZ, e->ldK));
    return ssad_slabsum(e->Z, e->Z, (long long)sZ, M, (long long)e->ldK * n, e->st);
}

/* ---- I instances of M channels (series i M .. i M + M - 1 of the engine are instance i) ---- */

/* Stacked CholQR of every instance: the Gram partials of its M channels are contiguous, so one
 * Cholesky job per instance sums all of them; every channel then takes its instance's R^{-1}. */
static int mssab_cholqr(ssa_engine *e, int I, int M, int n, double *colsum)
{
    const int B = I * M;
    const size_t sY = (size_t)e->ldL * e->kp;
    const int nch = (e->L + e->rows_L - 1) / e->rows_L;
    const size_t np = (size_t)n * (n + 1) / 2;
    CK(gram_ps(e, B, e->Y, sY, e->ldL, e->L, n, e->rows_L, 0, (size_t)nch * np));
    ssa_chol_job *cj = (ssa_chol_job *)calloc((size_t)I, sizeof(ssa_chol_job));
    ssa_rowmul_job *rj = (ssa_rowmul_job *)calloc((size_t)B, sizeof(ssa_rowmul_job));
    if (!cj || !rj)
    {
        free(cj);
        free(rj);
        return (int)cudaErrorMemoryAllocation;
    }
    for (int i = 0; i < I; i++)
    {
        cj[i].part = e->part + (size_t)i * M * nch * np;
        cj[i].Rinv = e->Rinv + (size_t)i * e->kp * e->kp;
        cj[i].status = e->status + i;
        cj[i].nchunks = M * nch;
        cj[i].n = n;
    }
    const int nqb = (e->L + SSA_ROWMUL_ROWS - 1) / SSA_ROWMUL_ROWS;
    for (int c = 0; c < B; c++)
    {
        ssa_rowmul_job *J = &rj[c];
        J->A = e->Y + (size_t)c * sY;
        J->C = e->Y + (size_t)c * sY;
        J->Bm64 = e->Rinv + (size_t)(c / M) * e->kp * e->kp;
        J->colsum = colsum ? colsum + (size_t)c * nqb * n : NULL;
        J->lda = e->ldL;
        J->ldc = e->ldL;
        J->m = e->L;
        J->n = n;
        J->p = n;
        J->ldb = n;
    }
    void *dc = ssae_push_jobs(e, cj, sizeof(ssa_chol_job) * I);
    void *dr = dc ? ssae_push_jobs(e, rj, sizeof(ssa_rowmul_job) * B) : NULL;
    free(cj);
    free(rj);
    if (!dc || !dr)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_CHOL);
    int rc = ssad_chol((const ssa_chol_job *)dc, I, e->st);
    ssae_prof_end(e);
    CK(rc);
    ssae_prof_begin(e, SSAK_ROWMUL);
    rc = ssad_rowmul((const ssa_rowmul_job *)dr, B, e->L, n, e->st);
    ssae_prof_end(e);
    return rc;
}

/* Scratch of the stacked forward sweeps: one spectrum of ldS floats per block column of every
 * instance. */
static int mssab_scratch(ssa_engine *e, int I)
{
    const size_t need = (size_t)I * e->kp * (size_t)e->ldS;
    if (need <= e->zs_cap)
        return 0;
    ssae_dfree(e, e->Zs);
    e->Zs = NULL;
    e->zs_cap = 0;
    CK(ssae_dalloc(e, (void **)&e->Zs, sizeof(float) * need));
    e->zs_cap = need;
    return 0;
}

/* The stacked forward sweeps run fused for the single-CTA transform lengths: each block column
 * is transformed once for all channels. */
static int mssab_fused(const ssa_engine *e, int M) { return M > 1 && e->logh <= SSA_ONE_CTA_MAX_LOGH && !ssad_cl14(); }

/* Z_{i M} = sum_m H_{i,m}^T Y_{i,m} for every instance. Fused: the channels' conj-products added
 * into one accumulator per instance column (a launch per channel, in channel order), then one
 * inverse transform per column; else per-channel adjoints into their Z slots and a fixed-order
 * channel sum per instance into its first channel's slot. */
static int mssab_adjoint(ssa_engine *e, int I, int M, int n)
{
    const size_t sY = (size_t)e->ldL * e->kp, sZ = (size_t)e->ldK * e->kp;
    if (!mssab_fused(e, M))
    {
        CK(corr_io(e, I * M, n, 1, e->Y, sY, e->ldL, e->Z, sZ, e->ldK));
        return ssad_slabsum_batch(e->Z, e->Z, (long long)sZ, M, (long long)e->ldK * n, I, (long long)M * sZ, e->st);
    }
    CK(mssab_scratch(e, I));
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)(M + 1) * I, sizeof(ssa_col_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int m = 0; m <= M; m++)
        for (int i = 0; i < I; i++)
        {
            ssa_col_job *J = &jobs[(size_t)m * I + i];
            J->spec = e->Zs + (size_t)i * e->kp * e->ldS;
            J->ld_spec = e->ldS;
            J->ncols = n;
            J->N = e->N;
            J->L = e->L;
            J->K = e->K;
            if (m < M)
            {
                J->in = e->Y + (size_t)(i * M + m) * sY;
                J->ld_in = e->ldL;
                J->n_in = e->L;
                J->X = e->X + (size_t)(i * M + m) * e->ldS;
            }
            else
            {
                J->out = e->Z + (size_t)i * M * sZ;
                J->ld_out = e->ldK;
                J->n_out = e->K;
            }
        }
    ssa_col_job *d = (ssa_col_job *)ssae_push_jobs(e, jobs, sizeof(ssa_col_job) * (size_t)(M + 1) * I);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_CORR);
    int rc = 0;
    for (int m = 0; m < M && !rc; m++)
        rc = ssad_corr_acc(d + (size_t)m * I, I, n, e->logh, m == 0, e->st);
    if (!rc)
        rc = ssad_corr_spec(d + (size_t)M * I, I, n, e->logh, e->st);
    ssae_prof_end(e);
    return rc;
}

/* Y_{i,m} = H_{i,m} Z_{i M}: every channel of an instance reads the instance's block (fused: the
 * block's columns transformed once, then every channel's product and inverse transform). */
static int mssab_forward(ssa_engine *e, int I, int M, int n)
{
    const size_t sY = (size_t)e->ldL * e->kp, sZ = (size_t)e->ldK * e->kp;
    const int B = I * M;
    const int fused = mssab_fused(e, M);
    if (fused)
    {
        CK(mssab_scratch(e, I));
        ssa_col_job *sj = (ssa_col_job *)calloc((size_t)I, sizeof(ssa_col_job));
        if (!sj)
            return (int)cudaErrorMemoryAllocation;
        for (int i = 0; i < I; i++)
        {
            ssa_col_job *J = &sj[i];
            J->in = e->Z + (size_t)i * M * sZ;
            J->ld_in = e->ldK;
            J->n_in = e->K;
            J->spec = e->Zs + (size_t)i * e->kp * e->ldS;
            J->ld_spec = e->ldS;
            J->ncols = n;
            J->N = e->N;
            J->L = e->L;
            J->K = e->K;
        }
        void *d = ssae_push_jobs(e, sj, sizeof(ssa_col_job) * I);
        free(sj);
        if (!d)
            return (int)cudaErrorMemoryAllocation;
        ssae_prof_begin(e, SSAK_CORR);
        int rc = ssad_spectrum((const ssa_col_job *)d, I, n, e->logh, e->st);
        ssae_prof_end(e);
        CK(rc);
    }
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)B, sizeof(ssa_col_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int c = 0; c < B; c++)
    {
        ssa_col_job *J = &jobs[c];
        J->in = e->Z + (size_t)(c / M) * M * sZ;
        J->ld_in = e->ldK;
        J->n_in = e->K;
        J->out = e->Y + (size_t)c * sY;
        J->ld_out = e->ldL;
        J->n_out = e->L;
        J->X = e->X + (size_t)c * e->ldS;
        J->spec = fused ? e->Zs + (size_t)(c / M) * e->kp * e->ldS : NULL;
        J->ld_spec = e->ldS;
        J->ncols = n;
        J->N = e->N;
        J->L = e->L;
        J->K = e->K;
    }
    void *d = ssae_push_jobs(e, jobs, sizeof(ssa_col_job) * B);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(e, SSAK_CORR);
    int rc = fused ? ssad_corr_spec((const ssa_col_job *)d, B, n, e->logh, e->st)
                   : ssad_corr((const ssa_col_job *)d, B, n, e->logh, e->st);
    ssae_prof_end(e);
    return rc;
}

int ssae_mssa_batch_decompose(ssa_engine *e, int I, int M, int kp, int k, int q, unsigned long long seed)
{
    const int B = I * M;
    if (I < 1 || M < 1 || B > e->B || kp < 1 || kp > e->kp || k < 1 || k > imin(kp, e->k))
        return (int)cudaErrorInvalidValue;
    const size_t sY = (size_t)e->ldL * e->kp, sZ = (size_t)e->ldK * e->kp;
    const int K = e->K;
    CK(cudaMemsetAsync(e->status, 0, sizeof(int) * I, e->st));
    /* start block of instance i (the device generator, seed mixed with the instance) in Z_{i M} */
    for (int i = 0; i < I; i++)
        CK(ssad_gaussian(e->Z + (size_t)i * M * sZ, e->ldK, K, kp, 0,
                         seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1)), e->st));
    CK(mssab_forward(e, I, M, kp));
    for (int it = 0; it < q; it++)
    {
        CK(mssab_cholqr(e, I, M, kp, NULL));
        CK(mssab_adjoint(e, I, M, kp));
        CK(cholqr_pass(e, I, e->Z, (size_t)M * sZ, e->ldK, K, kp, e->rows_K, NULL));
        CK(mssab_forward(e, I, M, kp));
    }
    CK(mssab_cholqr(e, I, M, kp, NULL));
    CK(mssab_cholqr(e, I, M, kp, e->qsum));
    CK(mssab_adjoint(e, I, M, kp));
    /* Rayleigh-Ritz per instance on B_i = Z_{i M} (its Gram partials at part + i * nchmax * np) */
    CK(gram(e, I, e->Z, (size_t)M * sZ, e->ldK, K, kp, e->rows_K, 0));
    {
        const int nchmax = imax(e->nch_L, imax(e->nch_K, e->nch_N));
        const size_t np = (size_t)e->kp * (e->kp + 1) / 2;
        const int nqb = (e->L + SSA_ROWMUL_ROWS - 1) / SSA_ROWMUL_ROWS;
        ssa_rr_job *J = (ssa_rr_job *)calloc((size_t)I, sizeof(ssa_rr_job));
        if (!J)
            return (int)cudaErrorMemoryAllocation;
        for (int i = 0; i < I; i++)
        {
            J[i].part = e->part + (size_t)i * nchmax * np;
            J[i].qsum = e->qsum + (size_t)i * M * nqb * kp;
            J[i].sigma = e->sigma + (size_t)i * M * e->k;
            J[i].Zu = e->Zu + (size_t)i * e->kp * e->k;
            J[i].Zv = e->Zv + (size_t)i * e->kp * e->k;
            J[i].status = e->status + i;
            J[i].nchunks = (K + e->rows_K - 1) / e->rows_K;
            J[i].nchunks_q = M * nqb;
            J[i].kp = kp;
            J[i].k = k;
        }
        void *d = ssae_push_jobs(e, J, sizeof(ssa_rr_job) * I);
        free(J);
        if (!d)
            return (int)cudaErrorMemoryAllocation;
        ssae_prof_begin(e, SSAK_RR);
        int rc = ssad_rr((const ssa_rr_job *)d, I, e->st);
        ssae_prof_end(e);
        CK(rc);
    }
    /* U_{i,m} = Q_{i,m} Zu_i for every channel; V_i = B_i Zv_i */
    {
        ssa_rowmul_job *rj = (ssa_rowmul_job *)calloc((size_t)(B + I), sizeof(ssa_rowmul_job));
        if (!rj)
            return (int)cudaErrorMemoryAllocation;
        for (int c = 0; c < B; c++)
        {
            ssa_rowmul_job *R = &rj[c];
            R->A = e->Y + (size_t)c * sY;
            R->C = e->Y + (size_t)c * sY;
            R->Bm = e->Zu + (size_t)(c / M) * e->kp * e->k;
            R->lda = R->ldc = e->ldL;
            R->m = e->L;
            R->n = kp;
            R->p = k;
            R->ldb = kp;
        }
        void *d = ssae_push_jobs(e, rj, sizeof(ssa_rowmul_job) * B);
        if (!d)
        {
            free(rj);
            return (int)cudaErrorMemoryAllocation;
        }
        ssae_prof_begin(e, SSAK_ROWMUL);
        int rc = ssad_rowmul((const ssa_rowmul_job *)d, B, e->L, kp, e->st);
        ssae_prof_end(e);
        CK(rc);
        for (int i = 0; i < I; i++)
        {
            ssa_rowmul_job *R = &rj[B + i];
            R->A = e->Z + (size_t)i * M * sZ;
            R->C = e->Z + (size_t)i * M * sZ;
            R->Bm = e->Zv + (size_t)i * e->kp * e->k;
            R->lda = R->ldc = e->ldK;
            R->m = K;
            R->n = kp;
            R->p = k;
            R->ldb = kp;
        }
        d = ssae_push_jobs(e, rj + B, sizeof(ssa_rowmul_job) * I);
        free(rj);
        if (!d)
            return (int)cudaErrorMemoryAllocation;
        ssae_prof_begin(e, SSAK_ROWMUL);
        rc = ssad_rowmul((const ssa_rowmul_job *)d, I, K, kp, e->st);
        ssae_prof_end(e);
        CK(rc);
    }
    return 0;
}

int ssae_mssa_decompose(ssa_engine *e, int M, int kp, int k, int q, const float *d_omega, unsigned long long seed)
{
    if (M < 1 || M > e->B || kp < 1 || kp > e->kp || k < 1 || k > imin(kp, e->k))
        return (int)cudaErrorInvalidValue;
    const size_t sY = (size_t)e->ldL * e->kp, sZ = (size_t)e->ldK * e->kp;
    const int K = e->K;
    CK(cudaMemsetAsync(e->status, 0, sizeof(int) * M, e->st));
    /* Omega (shared by every channel) in Z_0 */
    if (d_omega && d_omega != e->Z)
        CK(cudaMemcpy2DAsync(e->Z, sizeof(float) * e->ldK, d_omega, sizeof(float) * e->ldK, sizeof(float) * K, kp,
                             cudaMemcpyDeviceToDevice, e->st));
    else if (!d_omega)
        CK(ssad_gaussian(e->Z, e->ldK, K, kp, 0, seed, e->st));
    /* Y_m = H_m Omega */
    CK(corr_io(e, M, kp, 0, e->Z, 0, e->ldK, e->Y, sY, e->ldL));
    for (int it = 0; it < q; it++)
    {
        CK(mssa_cholqr(e, M, kp, NULL));
        CK(mssa_adjoint(e, M, kp));
        CK(cholqr_pass(e, 1, e->Z, sZ, e->ldK, K, kp, e->rows_K, NULL));
        CK(corr_io(e, M, kp, 0, e->Z, 0, e->ldK, e->Y, sY, e->ldL));
    }
    CK(mssa_cholqr(e, M, kp, NULL));
    CK(mssa_cholqr(e, M, kp, e->qsum));
    /* B = sum_m H_m^T Q_m, Rayleigh-Ritz on B^T B */
    CK(mssa_adjoint(e, M, kp));
    CK(gram(e, 1, e->Z, sZ, e->ldK, K, kp, e->rows_K, 0));
    {
        ssa_rr_job J;
        memset(&J, 0, sizeof(J));
        J.part = e->part;
        J.qsum = e->qsum;
        J.sigma = e->sigma;
        J.Zu = e->Zu;
        J.Zv = e->Zv;
        J.status = e->status;
        J.nchunks = (K + e->rows_K - 1) / e->rows_K;
        J.nchunks_q = M * ((e->L + SSA_ROWMUL_ROWS - 1) / SSA_ROWMUL_ROWS);
        J.kp = kp;
        J.k = k;
        void *d = ssae_push_jobs(e, &J, sizeof(J));
        if (!d)
            return (int)cudaErrorMemoryAllocation;
        ssae_prof_begin(e, SSAK_RR);
        int rc = ssad_rr((const ssa_rr_job *)d, 1, e->st);
        ssae_prof_end(e);
        CK(rc);
    }
    /* U_m = Q_m Zu for every channel; V = B Zv into Z_0 */
    CK(rowmul(e, M, e->Y, sY, e->ldL, e->L, kp, e->Zu, 0, kp, k, e->Y, sY, e->ldL, NULL, NULL));
    CK(rowmul(e, 1, e->Z, sZ, e->ldK, K, kp, e->Zv, 0, kp, k, e->Z, sZ, e->ldK, NULL, NULL));
    /* every channel's V slot gets V (the per-channel spectra of the reconstruction use them) */
    for (int m = 1; m < M; m++)
    {
        CK(cudaMemcpy2DAsync(e->Z + (size_t)m * sZ, sizeof(float) * e->ldK, e->Z, sizeof(float) * e->ldK,
                             sizeof(float) * K, k, cudaMemcpyDeviceToDevice, e->st));
        CK(cudaMemcpyAsync(e->sigma + (size_t)m * e->k, e->sigma, sizeof(double) * k, cudaMemcpyDeviceToDevice,
                           e->st));
    }
    return 0;
}
