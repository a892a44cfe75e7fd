/*
 * Uneven batches: B series of different lengths N[s], windows L[s] and ranks k[s] through the
 * randomized pipeline (decomposition with q power iterations, all k[s] elementary
 * reconstructions, W-correlation, group sums) in one launch per stage per FFT-length bucket.
 *
 * The kernels are job-driven (every job carries its own dims, pointers and leading dims, and
 * CTAs beyond a job's columns or rows return at once), so a bucket's launch covers series of any
 * shape whose FFT length M = 2^(logh+1) is the bucket's. Each bucket owns a CUDA stream; the
 * buckets of one run overlap on the device and join the batch's main stream at the end.
 *
 * Per-series layout inside a bucket (element offsets computed on the host per run):
 *   X     [i * ldS]            signal spectrum (bucket-uniform ldS)
 *   Y     [oY]  ldL x kp       range finder block, then U
 *   Z     [oZ]  ldK x kp       Z block, then B, then V
 *   part  [opart]              FP64 Gram partials, max(nch) * kp (kp + 1) / 2
 *   qsum  [oqsum] nq x kp      column-sum partials of the final Q (sign rule)
 *   R     [oR]  kp x kp        inverse Cholesky factor R^{-1} (FP64) of the last CholQR pass
 *   Zu/Zv [oZu] kp x k         Ritz rotations
 *   recon [orecon] k x ldN     elementary reconstructions
 *   norm2 [onorm] k
 *   Us    [ospec] k x ldS      spectra of sigma_i u_i (one-buffer reconstruction only)
 * Batch-level packed arrays (series order): x (sum N), sigma (sum k), W (sum k^2),
 * groups (n_groups * sum N), status (B).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <cuda_runtime_api.h>

#include "ssa_engine.h"
#include "ssa_ragged_int.h"
#include "../../include/ssa_opt.h"

#define CK(x)                  \
    do                         \
    {                          \
        int _e = (int)(x);     \
        if (_e != 0)           \
            return _e;         \
    } while (0)

/* buckets are indexed by FFT size code (ssad_fft_code_for): logh 4..16 and the two lengths
 * 3 * 2^13, 3 * 2^14 between the cluster powers of two */
#define RB_MIN_LOGH 4
#define RB_NB SSA_FFT_NCODES
_Static_assert(RB_NB == SSAR_NB, "bucket count of the internal header");

typedef struct
{
    int src; /* index in the batch */
    int N, L, K, kp, k;
    long long ldL, ldK, ldN;
    int rows_L, rows_K, rows_N, nch_L, nch_K, nch_N, nq;
    int rows_W, nch_W; /* W-correlation Gram chunks (tensor-core path: longer chunks) */
    int code;          /* FFT size code (a multi-length bucket holds several) */
    long long ldS;     /* floats of its signal spectrum (2 (H + 1) rounded) */
    size_t oX;         /* offset of its signal spectrum in the bucket's X */
    int wantW;         /* W-correlation requested for this series */
    int nelem;         /* elementary reconstructions computed: k with W, else those the groups use */
    /* follow-up runs: the series' resident factors (U ld ldL, V ld ldK, sigma) and its own group
     * (device indices gx[0..gn), largest index gmax); NULL outside follow-up runs */
    const float *Ux, *Vx;
    const double *sx;
    const int *gx;
    int gn, gmax;
    size_t oY, oZ, opart, oqsum, oR, oZu, orecon, onorm, ospec;
    size_t ox, osig, oW, ogrp;
} rser;

typedef struct
{
    ssa_engine e; /* stream, job arena, profiler */
    int live;
    int logh;
    int multi; /* series of every size code SSA_MULTI_MIN_LOGH .. SSA_MULTI_MAX_LOGH: the sweeps run
                  as one persistent launch over (series, column group, length) tiles */
    long long ldS;
    int nb, cap_nb;
    rser *sd;
    /* views into the batch's device arena for the current run */
    float *X, *Y, *Z, *Zu, *Zv, *recon, *Us;
    double *R; /* R^{-1} of the last CholQR pass, FP64 */
    double *part, *qsum, *norm2;
    size_t sz[11]; /* bytes of X, Y, Z, part, qsum, R, Zu, Zv, recon, norm2, Us for the run */
    int *status_base; /* the batch's status words (indexed by series) */
    cudaEvent_t done;
    float *bsplit;     /* tensor-core row products: split parts of the small factors, per series */
    size_t bsplit_cap; /* floats */
} rbucket;

struct ssa_rbatch
{
    int p, q, n_groups, total_idx;
    int grp_need; /* highest component index named by a group, plus one */
    int *d_gidx, *d_goff;
    rbucket bk[RB_NB];
    cudaStream_t main;
    cudaEvent_t ev_in;
    int prof;
    double *d_xs;
    size_t c_xs;
    /* one device arena holds every bucket buffer and the packed outputs of a run */
    char *arena;
    size_t arena_cap;
    double *sigma, *W, *groups;
    int *status;
    int B;
    size_t n_x, n_sig, n_W, n_grp;
    size_t *h_off; /* 4 B offsets of the last run: x, sigma, W, groups */
    /* optional per-run extensions (ssar_run_enqueue_ex) */
    const unsigned long long *cur_seeds; /* per-series generator seeds, or NULL */
    double *const *cur_lrf;              /* per-series LRF destinations, or NULL */
    const unsigned char *cur_wmask;      /* per-series "W-correlation wanted", or NULL = all */
    int lrf_slot, n_lrf_group, lrf_gmax;
    int *d_lrf_group;
    int *lrf_status;
    /* CUDA graphs of whole runs: a run whose launch signature was also the previous run's is
     * captured, and later runs with that signature replay the graph (job tables restored into
     * the staging areas, seeds through d_seeds) */
    struct rgraph
    {
        unsigned long long sig, stamp;
        unsigned long long kernels; /* kernel launches the graph holds */
        cudaGraphExec_t exec;
        char *snap[RB_NB];
        size_t snap_n[RB_NB];
    } graphs[4];
    unsigned long long last_sig, gstamp;
    int graphs_on, graph_pending;
    cudaEvent_t ev_graph;
    long long n_captures, n_replays;
    unsigned long long *h_seeds, *d_seeds;
    size_t c_seeds;
    /* follow-up runs (ssar_run_followup): given factors, per-series groups, no decomposition */
    int followup;
    const float *const *fu_U, *const *fu_V;
    const double *const *fu_sig;
    const int *fu_goff;
    int *h_fu_gidx, *d_fu_gidx;
    size_t c_fu_gidx;
};

/* The uneven batches run one stream per FFT-length bucket, and the server several batches at
 * once. With the runtime's default of 8 hardware work queues per device, streams beyond 8 share
 * queues, so a small batch's kernels wait in line behind a large batch's (measured: p99 latency
 * of 45-120 ms at 2k-5k requests/s, against 3-7 ms with 32 queues). Ask for 32 unless the process
 * chose its own value; this only takes effect when no CUDA context exists yet as the library is
 * loaded. */
__attribute__((constructor)) static void ssar_hw_queues(void) { setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0); }

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

/* Series whose transforms fit one CTA of 512 threads (size codes SSA_MULTI_MIN_LOGH ..
 * SSA_MULTI_MAX_LOGH) share one bucket whose correlation sweeps are one persistent launch
 * (ssad_corr_multi); off, every size code is a bucket of its own. */
static int g_multi = 1;
void ssa_b200_set_multi_length(int on) { g_multi = on != 0; }
int ssa_b200_multi_length(void) { return g_multi; }

struct rgraph;
static void graph_free(struct rgraph *g);

static int bucket_of(int code)
{
    return (g_multi && code >= SSA_MULTI_MIN_LOGH && code <= SSA_MULTI_MAX_LOGH) ? SSA_MULTI_MAX_LOGH : code;
}
static long long round4(long long v) { return (v + 3) & ~3LL; }

/* Per-bucket launch parameters chosen by the autotuner (0 = the built-in heuristic): the CTA count
 * the Gram partial launches aim at for each FFT size code, and the CTAs per SM of the persistent
 * multi-length sweep. Host state only; set through ssa_b200_tune_set. */
static struct
{
    int gram_ctas[RB_NB];
    int multi_ctas_per_sm;
} g_tune;

int ssa_b200_tune_set(const int *gram_ctas, int n, int multi_ctas_per_sm)
{
    if (n < 0 || n > RB_NB || multi_ctas_per_sm < 0 || multi_ctas_per_sm > 2)
        return -1;
    for (int i = 0; i < RB_NB; i++)
    {
        const int v = (gram_ctas && i < n) ? gram_ctas[i] : 0;
        if (v < 0 || v > 65536)
            return -1;
        g_tune.gram_ctas[i] = v;
    }
    g_tune.multi_ctas_per_sm = multi_ctas_per_sm;
    return 0;
}

int ssa_b200_tune_get(int *gram_ctas, int n, int *multi_ctas_per_sm)
{
    for (int i = 0; i < n && i < RB_NB; i++)
        gram_ctas[i] = g_tune.gram_ctas[i];
    if (multi_ctas_per_sm)
        *multi_ctas_per_sm = g_tune.multi_ctas_per_sm;
    return RB_NB;
}

/* Rows per Gram partial for a block of m rows in a bucket of nb series with FFT size code
 * `code` (code < 0: the heuristic). */
static int gram_rows_for(int m, int nb, int code)
{
    /* about 1184 CTAs (eight per SM) over the bucket's series, or the tuned count */
    const int ctas = (code >= 0 && code < RB_NB && g_tune.gram_ctas[code] > 0) ? g_tune.gram_ctas[code] : 1184;
    int target = ctas / (nb > 0 ? nb : 1);
    if (target < 1)
        target = 1;
    int rows = (m + target - 1) / target;
    rows = ((rows + SSA_GRAM_CHUNK - 1) / SSA_GRAM_CHUNK) * SSA_GRAM_CHUNK;
    /* at least four staging chunks per CTA: fewer partials for the per-series kernels to sum
     * (their latency) when a launch holds few series */
    return imax(rows, 4 * SSA_GRAM_CHUNK);
}

static int gram_rows(int m, int nb) { return gram_rows_for(m, nb, -1); }

/* The library's stream-ordered memory pool on the current device: freed blocks stay cached in
 * it (release threshold at its maximum), so re-growing buffers costs no driver allocation. */
int ssar_bucket_index(int N) { return bucket_of(ssad_fft_code_for(N)); }

cudaStream_t ssar_bucket_stream(const ssa_rbatch *rb, int g)
{
    return (rb && g >= 0 && g < RB_NB && rb->bk[g].live && rb->bk[g].nb) ? rb->bk[g].e.st : NULL;
}

cudaMemPool_t ssar_pool(void)
{
    static cudaMemPool_t pools[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return NULL;
    if (!pools[dev])
    {
        struct cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess)
            return NULL;
        unsigned long long thr = ~0ULL;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        pools[dev] = pool;
    }
    return pools[dev];
}

/* Grow a device buffer to at least `need` elements of `elem` bytes (contents not kept), in
 * stream order on `st` (the stream that uses it), so that growing never waits for the device:
 * cudaFree would synchronise every stream, including other batches in flight. */
static int grow(void **p, size_t *cap, size_t need, size_t elem, cudaStream_t st)
{
    if (need <= *cap && *p)
        return 0;
    if (*p)
        cudaFreeAsync(*p, st);
    *p = NULL;
    *cap = 0;
    if (need == 0)
        return 0;
    size_t n = need + need / 8;
    cudaMemPool_t pool = ssar_pool();
    if (!pool)
        return (int)cudaErrorMemoryAllocation;
    CK(cudaMallocFromPoolAsync(p, n * elem, pool, st));
    *cap = n;
    return 0;
}

static void bucket_free(rbucket *b)
{
    if (!b->live)
        return;
    if (b->bsplit)
        cudaFreeAsync(b->bsplit, b->e.st);
    ssae_destroy(&b->e); /* stream, job arena, profiler events */
    if (b->done)
        cudaEventDestroy(b->done);
    free(b->sd);
    memset(b, 0, sizeof(*b));
}

void ssa_rbatch_destroy(ssa_rbatch *rb)
{
    if (rb && rb->h_fu_gidx)
        cudaFreeHost(rb->h_fu_gidx);
    if (rb && rb->d_fu_gidx)
        cudaFree(rb->d_fu_gidx);
    if (!rb)
        return;
    if (rb->main)
        cudaStreamSynchronize(rb->main);
    for (int i = 0; i < RB_NB; i++)
        bucket_free(&rb->bk[i]);
    void *bufs[] = {rb->d_gidx, rb->d_goff, rb->d_xs, rb->arena, rb->d_lrf_group};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); i++)
        if (bufs[i])
            cudaFree(bufs[i]);
    if (rb->ev_in)
        cudaEventDestroy(rb->ev_in);
    for (int i = 0; i < 4; i++)
        graph_free(&rb->graphs[i]);
    if (rb->ev_graph)
        cudaEventDestroy(rb->ev_graph);
    if (rb->h_seeds)
        cudaFreeHost(rb->h_seeds);
    if (rb->d_seeds)
        cudaFree(rb->d_seeds);
    if (rb->main)
        cudaStreamDestroy(rb->main);
    free(rb->h_off);
    free(rb);
    /* hand the pool's cached blocks back to the driver (blocks in use elsewhere stay) */
    cudaMemPool_t pool = ssar_pool();
    if (pool)
        cudaMemPoolTrimTo(pool, 0);
}

int ssa_rbatch_create(ssa_rbatch **out, int oversampling, int power_iters, const int *group_idx,
                      const int *group_sizes, int n_groups)
{
    if (!out || power_iters < 0 || n_groups < 0 || (n_groups > 0 && (!group_idx || !group_sizes)))
        return -1;
    *out = NULL;
    ssa_rbatch *rb = (ssa_rbatch *)calloc(1, sizeof(*rb));
    if (!rb)
        return -1;
    rb->p = oversampling <= 0 ? 8 : oversampling;
    rb->q = power_iters;
    rb->n_groups = n_groups;
    rb->graphs_on = 1;
    if (ssad_init_device() != 0 || cudaStreamCreateWithFlags(&rb->main, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&rb->ev_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&rb->ev_graph, cudaEventDisableTiming) != cudaSuccess)
    {
        ssa_rbatch_destroy(rb);
        return -1;
    }
    if (n_groups > 0)
    {
        int *off = (int *)malloc(sizeof(int) * (n_groups + 1));
        if (!off)
        {
            ssa_rbatch_destroy(rb);
            return -1;
        }
        off[0] = 0;
        for (int g = 0; g < n_groups; g++)
            off[g + 1] = off[g] + (group_sizes[g] > 0 ? group_sizes[g] : 0);
        rb->total_idx = off[n_groups];
        for (int i = 0; i < rb->total_idx; i++)
            rb->grp_need = imax(rb->grp_need, group_idx[i] + 1);
        int rc = cudaMalloc((void **)&rb->d_goff, sizeof(int) * (n_groups + 1)) != cudaSuccess;
        rc |= cudaMalloc((void **)&rb->d_gidx, sizeof(int) * (rb->total_idx > 0 ? rb->total_idx : 1)) != cudaSuccess;
        if (!rc)
            rc |= cudaMemcpy(rb->d_goff, off, sizeof(int) * (n_groups + 1), cudaMemcpyHostToDevice) != cudaSuccess;
        if (!rc && rb->total_idx > 0)
            rc |= cudaMemcpy(rb->d_gidx, group_idx, sizeof(int) * rb->total_idx, cudaMemcpyHostToDevice) !=
                  cudaSuccess;
        free(off);
        if (rc)
        {
            ssa_rbatch_destroy(rb);
            return -1;
        }
    }
    *out = rb;
    return 0;
}

static int bucket_setup(rbucket *b, int logh, int prof)
{
    if (!b->live)
    {
        CK(ssae_create_light(&b->e, 1 << 20, NULL));
        CK(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
        b->live = 1;
    }
    if (prof && !b->e.prof)
        CK(ssae_set_profiling(&b->e, 1));
    b->logh = logh; /* size code */
    b->ldS = round4(2LL * (ssad_fft_h(logh) + 1) + 2);
    return 0;
}

/* ---- stages ------------------------------------------------------------------------------ */

/* Series of the bucket with size code `code`, in bucket order (all of them for a one-code bucket). */
static int code_members(const rbucket *b, int code, int *idx)
{
    int n = 0;
    for (int i = 0; i < b->nb; i++)
        if (b->sd[i].code == code)
            idx[n++] = i;
    return n;
}

/* Launch `launch(jobs, n, code)` once per size code present in the bucket, each with the jobs of
 * that code's series (one launch for a one-code bucket). jobs holds one job per series. */
typedef int (*code_launch_fn)(rbucket *b, const void *d_jobs, int n, int maxc, int code);
static int per_code(rbucket *b, const void *jobs, size_t jsz, const int *maxc_of, code_launch_fn launch)
{
    if (!b->multi)
    {
        int maxc = 0;
        for (int i = 0; i < b->nb; i++)
            maxc = imax(maxc, maxc_of[i]);
        void *d = ssae_push_jobs(&b->e, jobs, jsz * b->nb);
        return d ? launch(b, d, b->nb, maxc, b->logh) : (int)cudaErrorMemoryAllocation;
    }
    int *idx = (int *)malloc(sizeof(int) * (size_t)b->nb);
    char *sub = (char *)malloc(jsz * (size_t)b->nb);
    if (!idx || !sub)
    {
        free(idx);
        free(sub);
        return (int)cudaErrorMemoryAllocation;
    }
    int rc = 0;
    for (int code = SSA_MULTI_MAX_LOGH; code >= SSA_MULTI_MIN_LOGH && !rc; code--)
    {
        const int n = code_members(b, code, idx);
        if (!n)
            continue;
        int maxc = 0;
        for (int j = 0; j < n; j++)
        {
            memcpy(sub + jsz * j, (const char *)jobs + jsz * idx[j], jsz);
            maxc = imax(maxc, maxc_of[idx[j]]);
        }
        void *d = ssae_push_jobs(&b->e, sub, jsz * n);
        rc = d ? launch(b, d, n, maxc, code) : (int)cudaErrorMemoryAllocation;
    }
    free(idx);
    free(sub);
    return rc;
}

static int launch_spectrum_code(rbucket *b, const void *d, int n, int maxc, int code)
{
    if (maxc <= 0)
        return 0;
    ssae_prof_begin(&b->e, SSAK_SPECTRUM);
    const int rc = ssad_spectrum((const ssa_col_job *)d, n, maxc, code, b->e.st);
    ssae_prof_end(&b->e);
    return rc;
}

static int launch_elem_code(rbucket *b, const void *d, int n, int maxc, int code)
{
    if (maxc <= 0)
        return 0;
    ssae_prof_begin(&b->e, SSAK_ELEM);
    const int rc = code > SSA_ELEM2_MAX_LOGH ? ssad_elem_recon1((const ssa_col_job *)d, n, maxc, code, b->e.st)
                                             : ssad_elem_recon((const ssa_col_job *)d, n, maxc, code, b->e.st);
    ssae_prof_end(&b->e);
    return rc;
}

static int r_spectrum(rbucket *b, const double *d_x)
{
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)b->nb, sizeof(ssa_col_job));
    int *ones = (int *)malloc(sizeof(int) * (size_t)b->nb);
    if (!jobs || !ones)
    {
        free(jobs);
        free(ones);
        return (int)cudaErrorMemoryAllocation;
    }
    for (int i = 0; i < b->nb; i++)
    {
        const rser *S = &b->sd[i];
        ssa_col_job *J = &jobs[i];
        J->in64 = d_x + S->ox;
        J->ld_in = S->N;
        J->n_in = S->N;
        J->spec = b->X + S->oX;
        J->ld_spec = S->ldS;
        J->ncols = 1;
        J->N = S->N;
        J->L = S->L;
        J->K = S->K;
        ones[i] = 1;
    }
    const int rc = per_code(b, jobs, sizeof(ssa_col_job), ones, launch_spectrum_code);
    free(jobs);
    free(ones);
    return rc;
}

/* adjoint 0: Y = H (Omega | Z); adjoint 1: Z = H^T Y. generate: Omega from the device generator,
 * series seed seeds[src] when given, else seed mixed with the batch position. */
static int r_sweep(rbucket *b, int adjoint, int generate, const unsigned long long *d_seeds)
{
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)b->nb, sizeof(ssa_col_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int i = 0; i < b->nb; i++)
    {
        const rser *S = &b->sd[i];
        ssa_col_job *J = &jobs[i];
        float *Ys = b->Y + S->oY, *Zs = b->Z + S->oZ;
        if (!adjoint)
        {
            if (generate)
            {
                J->in = NULL;
                J->seedp = d_seeds + S->src; /* read by the kernel: job tables stay run-invariant */
            }
            else
            {
                J->in = Zs;
                J->ld_in = S->ldK;
            }
            J->n_in = S->K;
            J->out = Ys;
            J->ld_out = S->ldL;
            J->n_out = S->L;
        }
        else
        {
            J->in = Ys;
            J->ld_in = S->ldL;
            J->n_in = S->L;
            J->out = Zs;
            J->ld_out = S->ldK;
            J->n_out = S->K;
        }
        J->X = b->X + S->oX;
        J->ncols = S->kp;
        J->N = S->N;
        J->L = S->L;
        J->K = S->K;
    }
    void *d = ssae_push_jobs(&b->e, jobs, sizeof(ssa_col_job) * b->nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    if (b->multi)
    {
        /* the work queue: (series, column group, length) tiles, longest lengths first, and its
         * head counter (zero, copied with the tiles) */
        int nt = 0;
        for (int i = 0; i < b->nb; i++)
        {
            const int g = ssad_multi_tile_cols(b->sd[i].code);
            nt += (b->sd[i].kp + g - 1) / g;
        }
        ssa_tile *tiles = (ssa_tile *)calloc((size_t)nt + 1, sizeof(ssa_tile));
        if (!tiles)
            return (int)cudaErrorMemoryAllocation;
        int t = 0;
        for (int code = SSA_MULTI_MAX_LOGH; code >= SSA_MULTI_MIN_LOGH; code--)
            for (int i = 0; i < b->nb; i++)
            {
                const rser *S = &b->sd[i];
                if (S->code != code)
                    continue;
                const int g = ssad_multi_tile_cols(code);
                for (int c0 = 0; c0 < S->kp; c0 += g)
                {
                    tiles[t].job = i;
                    tiles[t].c0 = c0;
                    tiles[t].logh = code;
                    t++;
                }
            }
        /* tiles[nt] is the zeroed counter slot */
        void *dt = ssae_push_jobs(&b->e, tiles, sizeof(ssa_tile) * ((size_t)nt + 1));
        free(tiles);
        if (!dt)
            return (int)cudaErrorMemoryAllocation;
        ssae_prof_begin(&b->e, SSAK_CORR);
        int nctas = 0;
        if (g_tune.multi_ctas_per_sm > 0)
        {
            int dev = 0, nsm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            nctas = g_tune.multi_ctas_per_sm * nsm;
        }
        int rc = ssad_corr_multi((const ssa_col_job *)d, (const ssa_tile *)dt, nt, (int *)((ssa_tile *)dt + nt),
                                 nctas, b->e.st);
        ssae_prof_end(&b->e);
        return rc;
    }
    /* one CTA (cluster) per live column: the series' kp differ (k + p), so a (columns, series)
     * grid would hold a third of its CTAs for columns beyond a series' kp */
    int nt = 0;
    for (int i = 0; i < b->nb; i++)
        nt += b->sd[i].kp;
    ssa_tile *tiles = (ssa_tile *)calloc((size_t)nt + 1, sizeof(ssa_tile));
    if (!tiles)
        return (int)cudaErrorMemoryAllocation;
    int t = 0;
    for (int i = 0; i < b->nb; i++)
        for (int c = 0; c < b->sd[i].kp; c++)
        {
            tiles[t].job = i;
            tiles[t].c0 = c;
            tiles[t].logh = b->logh;
            t++;
        }
    void *dt = ssae_push_jobs(&b->e, tiles, sizeof(ssa_tile) * (size_t)nt);
    free(tiles);
    if (!dt)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(&b->e, SSAK_CORR);
    int rc = ssad_corr_tiles((const ssa_col_job *)d, (const ssa_tile *)dt, nt, b->logh, b->e.st);
    ssae_prof_end(&b->e);
    return rc;
}

enum
{
    SIDE_L = 0, /* Y blocks, L x kp */
    SIDE_K = 1, /* Z blocks, K x kp */
    SIDE_N = 2  /* elementary reconstructions, N x k, weighted */
};

static int r_gram(rbucket *b, int side)
{
    const int tc = side == SIDE_N && ssad_wcorr_tc();
    ssa_gram_job *jobs = (ssa_gram_job *)calloc((size_t)b->nb, sizeof(ssa_gram_job));
    ssa_wgram_job *wjobs = tc ? (ssa_wgram_job *)calloc((size_t)b->nb, sizeof(ssa_wgram_job)) : NULL;
    if (!jobs || (tc && !wjobs))
    {
        free(jobs);
        free(wjobs);
        return (int)cudaErrorMemoryAllocation;
    }
    int maxch = 0, nj = 0;
    for (int i = 0; i < b->nb; i++)
    {
        const rser *S = &b->sd[i];
        if (side == SIDE_N && !S->wantW)
            continue;
        ssa_gram_job *J = &jobs[nj];
        if (side == SIDE_L)
        {
            J->A = b->Y + S->oY;
            J->ld = S->ldL;
            J->m = S->L;
            J->n = S->kp;
            J->rows_per_cta = S->rows_L;
            maxch = imax(maxch, S->nch_L);
        }
        else if (side == SIDE_K)
        {
            J->A = b->Z + S->oZ;
            J->ld = S->ldK;
            J->m = S->K;
            J->n = S->kp;
            J->rows_per_cta = S->rows_K;
            maxch = imax(maxch, S->nch_K);
        }
        else
        {
            J->A = b->recon + S->orecon;
            J->ld = S->ldN;
            J->m = S->N;
            J->n = S->k;
            J->rows_per_cta = S->rows_W;
            J->weighted = 1;
            maxch = imax(maxch, S->nch_W);
        }
        J->part = b->part + S->opart;
        J->N = S->N;
        J->L = S->L;
        J->K = S->K;
        if (tc)
        {
            wjobs[nj].g = *J;
            wjobs[nj].status = b->status_base + S->src;
        }
        nj++;
    }
    if (nj == 0)
    {
        free(jobs);
        free(wjobs);
        return 0;
    }
    void *d = tc ? ssae_push_jobs(&b->e, wjobs, sizeof(ssa_wgram_job) * nj)
                 : ssae_push_jobs(&b->e, jobs, sizeof(ssa_gram_job) * nj);
    free(jobs);
    free(wjobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(&b->e, side == SIDE_N ? SSAK_WGRAM : SSAK_GRAM);
    int rc = tc ? ssad_gram_tc((const ssa_wgram_job *)d, nj, maxch, b->e.st)
                : ssad_gram((const ssa_gram_job *)d, nj, maxch, side == SIDE_N, b->e.st);
    ssae_prof_end(&b->e);
    return rc;
}

static int r_chol(rbucket *b, int side, int *status)
{
    ssa_chol_job *jobs = (ssa_chol_job *)calloc((size_t)b->nb, sizeof(ssa_chol_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int i = 0; i < b->nb; i++)
    {
        const rser *S = &b->sd[i];
        ssa_chol_job *J = &jobs[i];
        J->part = b->part + S->opart;
        J->Rinv = b->R + S->oR;
        J->status = status + S->src;
        J->nchunks = side == SIDE_L ? S->nch_L : S->nch_K;
        J->n = S->kp;
    }
    void *d = ssae_push_jobs(&b->e, jobs, sizeof(ssa_chol_job) * b->nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(&b->e, SSAK_CHOL);
    int rc = ssad_chol((const ssa_chol_job *)d, b->nb, b->e.st);
    ssae_prof_end(&b->e);
    return rc;
}

/* trsm: A = A R^{-1} in place (column-sum partials into qsum when `colsum`);
 * else A[:, :k] = A Zrot (U = Q Zu on the L side, V = B Zv on the K side). */
static int r_rowmul(rbucket *b, int side, int trsm, int colsum)
{
    ssa_rowmul_job *jobs = (ssa_rowmul_job *)calloc((size_t)b->nb, sizeof(ssa_rowmul_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    int maxm = 0, maxn = 0;
    for (int i = 0; i < b->nb; i++)
    {
        const rser *S = &b->sd[i];
        ssa_rowmul_job *J = &jobs[i];
        float *A = side == SIDE_L ? b->Y + S->oY : b->Z + S->oZ;
        const long long ld = side == SIDE_L ? S->ldL : S->ldK;
        const int m = side == SIDE_L ? S->L : S->K;
        J->A = A;
        J->C = A;
        J->lda = ld;
        J->ldc = ld;
        J->m = m;
        J->n = S->kp;
        J->ldb = S->kp;
        if (trsm)
        {
            J->Bm64 = b->R + S->oR;
            J->p = S->kp;
            J->colsum = colsum ? b->qsum + S->oqsum : NULL;
        }
        else
        {
            J->Bm = (side == SIDE_L ? b->Zu : b->Zv) + S->oZu;
            J->p = S->k;
        }
        maxm = imax(maxm, m);
        maxn = imax(maxn, S->kp);
    }
    const int tc = ssad_rowmul_tc_on();
    if (tc)
    {
        const int rc = grow((void **)&b->bsplit, &b->bsplit_cap, (size_t)b->nb * SSA_ROWMUL_BSPLIT_FLOATS, sizeof(float),
                            b->e.st);
        if (rc)
        {
            free(jobs);
            return rc;
        }
        for (int i = 0; i < b->nb; i++)
            jobs[i].Bsplit = b->bsplit + (size_t)i * SSA_ROWMUL_BSPLIT_FLOATS;
    }
    void *d = ssae_push_jobs(&b->e, jobs, sizeof(ssa_rowmul_job) * b->nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(&b->e, SSAK_ROWMUL);
    int rc = tc ? ssad_rowmul_tc((const ssa_rowmul_job *)d, b->nb, maxm, maxn, b->e.st)
                : ssad_rowmul((const ssa_rowmul_job *)d, b->nb, maxm, maxn, b->e.st);
    ssae_prof_end(&b->e);
    return rc;
}

static int r_cholqr(rbucket *b, int side, int colsum, int *status)
{
    CK(r_gram(b, side));
    CK(r_chol(b, side, status));
    return r_rowmul(b, side, 1, colsum);
}

static int r_rr(rbucket *b, double *sigma, int *status)
{
    ssa_rr_job *jobs = (ssa_rr_job *)calloc((size_t)b->nb, sizeof(ssa_rr_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    for (int i = 0; i < b->nb; i++)
    {
        const rser *S = &b->sd[i];
        ssa_rr_job *J = &jobs[i];
        J->part = b->part + S->opart;
        J->qsum = b->qsum + S->oqsum;
        J->sigma = sigma + S->osig;
        J->Zu = b->Zu + S->oZu;
        J->Zv = b->Zv + S->oZu;
        J->status = status + S->src;
        J->nchunks = S->nch_K;
        J->nchunks_q = S->nq;
        J->kp = S->kp;
        J->k = S->k;
    }
    void *d = ssae_push_jobs(&b->e, jobs, sizeof(ssa_rr_job) * b->nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(&b->e, SSAK_RR);
    int rc = ssad_rr((const ssa_rr_job *)d, b->nb, b->e.st);
    ssae_prof_end(&b->e);
    return rc;
}

static int r_elem(rbucket *b, const double *sigma)
{
    const int one = b->logh > SSA_ELEM2_MAX_LOGH; /* one-code buckets only: multi-length codes are <= 13 */
    ssa_col_job *jobs = (ssa_col_job *)calloc((size_t)b->nb, sizeof(ssa_col_job));
    int *ncols = (int *)malloc(sizeof(int) * (size_t)b->nb);
    if (!jobs || !ncols)
    {
        free(jobs);
        free(ncols);
        return (int)cudaErrorMemoryAllocation;
    }
    int maxk = 0;
    for (int i = 0; i < b->nb; i++)
    {
        ncols[i] = b->sd[i].nelem;
        maxk = imax(maxk, ncols[i]);
    }
    if (maxk == 0)
    {
        free(jobs);
        free(ncols);
        return 0;
    }
    int rc = 0;
    if (one)
    {
        /* spectra of sigma_i u_i first; the reconstruction kernel then holds one FFT buffer */
        for (int i = 0; i < b->nb; i++)
        {
            const rser *S = &b->sd[i];
            ssa_col_job *J = &jobs[i];
            J->in = S->Ux ? S->Ux : b->Y + S->oY;
            J->ld_in = S->ldL;
            J->n_in = S->L;
            J->scale = S->sx ? S->sx : sigma + S->osig;
            J->spec = b->Us + S->ospec;
            J->ld_spec = S->ldS;
            J->ncols = S->nelem;
        }
        rc = per_code(b, jobs, sizeof(ssa_col_job), ncols, launch_spectrum_code);
        memset(jobs, 0, sizeof(ssa_col_job) * b->nb);
    }
    for (int i = 0; i < b->nb && !rc; i++)
    {
        const rser *S = &b->sd[i];
        ssa_col_job *J = &jobs[i];
        J->in = S->Ux ? S->Ux : b->Y + S->oY;
        J->ld_in = S->ldL;
        J->n_in = S->L;
        J->in2 = S->Vx ? S->Vx : b->Z + S->oZ;
        J->ld_in2 = S->ldK;
        J->n_in2 = S->K;
        J->scale = S->sx ? S->sx : sigma + S->osig;
        J->out = b->recon + S->orecon;
        J->ld_out = S->ldN;
        J->norm2 = b->norm2 + S->onorm;
        J->ncols = S->nelem;
        J->N = S->N;
        J->L = S->L;
        J->K = S->K;
        if (one)
        {
            J->spec = b->Us + S->ospec;
            J->ld_spec = S->ldS;
        }
    }
    if (!rc)
        rc = per_code(b, jobs, sizeof(ssa_col_job), ncols, launch_elem_code);
    free(jobs);
    free(ncols);
    return rc;
}

static int r_wcorr(rbucket *b, double *W)
{
    CK(r_gram(b, SIDE_N));
    ssa_wfin_job *jobs = (ssa_wfin_job *)calloc((size_t)b->nb, sizeof(ssa_wfin_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    int nj = 0;
    for (int i = 0; i < b->nb; i++)
    {
        const rser *S = &b->sd[i];
        if (!S->wantW)
            continue;
        jobs[nj].part = b->part + S->opart;
        jobs[nj].W = W + S->oW;
        jobs[nj].nchunks = S->nch_W;
        jobs[nj].k = S->k;
        nj++;
    }
    if (nj == 0)
    {
        free(jobs);
        return 0;
    }
    void *d = ssae_push_jobs(&b->e, jobs, sizeof(ssa_wfin_job) * nj);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(&b->e, SSAK_WFIN);
    int rc = ssad_wfin((const ssa_wfin_job *)d, nj, b->e.st);
    ssae_prof_end(&b->e);
    return rc;
}

static int r_gsum(rbucket *b, ssa_rbatch *rb)
{
    ssa_rgsum_job *jobs = (ssa_rgsum_job *)calloc((size_t)b->nb, sizeof(ssa_rgsum_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    int maxN = 0;
    for (int i = 0; i < b->nb; i++)
    {
        const rser *S = &b->sd[i];
        jobs[i].recon = b->recon + S->orecon;
        jobs[i].ld_recon = S->ldN;
        jobs[i].out = rb->groups + S->ogrp;
        jobs[i].N = S->N;
        jobs[i].k = S->nelem; /* covers every grouped component below k */
        jobs[i].gidx = S->gx;
        jobs[i].gn = S->gn;
        maxN = imax(maxN, S->N);
    }
    void *d = ssae_push_jobs(&b->e, jobs, sizeof(ssa_rgsum_job) * b->nb);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(&b->e, SSAK_GSUM);
    int rc = ssad_group_sum_ragged((const ssa_rgsum_job *)d, b->nb, maxN, rb->d_gidx, rb->d_goff, rb->n_groups,
                                   b->e.st);
    ssae_prof_end(&b->e);
    return rc;
}

/* LRF coefficients and reconstruction tail of the forecast group (group slot rb->lrf_slot) into
 * the per-series destinations: R (L-1), tail (L-1), verticality (1) doubles. */
static int r_lrf(rbucket *b, ssa_rbatch *rb)
{
    ssa_lrf_job *jobs = (ssa_lrf_job *)calloc((size_t)b->nb, sizeof(ssa_lrf_job));
    if (!jobs)
        return (int)cudaErrorMemoryAllocation;
    int n = 0;
    for (int i = 0; i < b->nb; i++)
    {
        const rser *S = &b->sd[i];
        double *dst = rb->cur_lrf[S->src];
        const int gmax = S->gx ? S->gmax : rb->lrf_gmax;
        if (!dst || gmax >= S->k || gmax < 0)
            continue;
        ssa_lrf_job *J = &jobs[n++];
        J->U = S->Ux ? S->Ux : b->Y + S->oY;
        J->ld = S->ldL;
        J->group = S->gx ? S->gx : rb->d_lrf_group;
        J->n_group = S->gx ? S->gn : rb->n_lrf_group;
        J->recon = rb->groups + S->ogrp + (size_t)(S->gx ? 0 : rb->lrf_slot) * S->N;
        J->R = dst;
        J->buf = dst + (S->L - 1);
        J->out = NULL;
        J->verticality = dst + 2 * (size_t)(S->L - 1);
        J->status = rb->lrf_status + S->src;
        J->L = S->L;
        J->N = S->N;
        J->h = 0;
        J->k = S->k;
    }
    if (!n)
    {
        free(jobs);
        return 0;
    }
    void *d = ssae_push_jobs(&b->e, jobs, sizeof(ssa_lrf_job) * n);
    free(jobs);
    if (!d)
        return (int)cudaErrorMemoryAllocation;
    ssae_prof_begin(&b->e, SSAK_LRF);
    int rc = ssad_lrf((const ssa_lrf_job *)d, n, b->e.st);
    ssae_prof_end(&b->e);
    return rc;
}

/* Whole pipeline of one bucket on its stream (the stage order of ssae_decompose,
 * ssae_elem_recon, ssae_wcorr and the batch group sums). */
static int bucket_run(rbucket *b, ssa_rbatch *rb, const double *d_x, unsigned long long seed)
{
    CK(r_spectrum(b, d_x));
    CK(r_sweep(b, 0, 1, rb->d_seeds));
    for (int it = 0; it < rb->q; it++)
    {
        CK(r_cholqr(b, SIDE_L, 0, rb->status));
        CK(r_sweep(b, 1, 0, NULL));
        CK(r_cholqr(b, SIDE_K, 0, rb->status));
        CK(r_sweep(b, 0, 0, NULL));
    }
    CK(r_cholqr(b, SIDE_L, 0, rb->status));
    CK(r_cholqr(b, SIDE_L, 1, rb->status));
    CK(r_sweep(b, 1, 0, NULL));
    CK(r_gram(b, SIDE_K));
    CK(r_rr(b, rb->sigma, rb->status));
    CK(r_rowmul(b, SIDE_L, 0, 0));
    CK(r_rowmul(b, SIDE_K, 0, 0));
    CK(r_elem(b, rb->sigma));
    CK(r_wcorr(b, rb->W));
    if (rb->n_groups > 0)
        CK(r_gsum(b, rb));
    if (rb->cur_lrf && rb->n_lrf_group > 0 && rb->n_groups > 0)
        CK(r_lrf(b, rb));
    return 0;
}

/* Follow-up pipeline of one bucket: elementary reconstructions of the series' resident factors
 * (components 0 .. gmax), the sum of its own group, and the group's LRF where asked for. */
static int bucket_followup(rbucket *b, ssa_rbatch *rb)
{
    CK(r_elem(b, NULL));
    CK(r_gsum(b, rb));
    if (rb->cur_lrf)
        CK(r_lrf(b, rb));
    return 0;
}

int ssa_b200_fft_size_code(int N) { return N >= 1 ? ssad_fft_code_for(N) : -1; }
void ssa_b200_set_cluster32k(int on) { ssad_set_cl14(on); }
int ssa_b200_cluster32k(void) { return ssad_cl14(); }

int ssa_b200_fft_length(int N)
{
    const int code = N >= 1 ? ssad_fft_code_for(N) : -1;
    return code < 0 ? -1 : 2 * ssad_fft_h(code);
}

/* Device arena of at least `bytes` (stream-ordered on the main stream after the previous run). */
int ssa_rbatch_reserve(ssa_rbatch *rb, size_t bytes)
{
    if (!rb)
        return -1;
    if (bytes <= rb->arena_cap)
        return 0;
    cudaMemPool_t pool = ssar_pool();
    if (!pool)
        return -1;
    if (rb->arena)
        cudaFreeAsync(rb->arena, rb->main);
    rb->arena = NULL;
    rb->arena_cap = 0;
    if (cudaMallocFromPoolAsync((void **)&rb->arena, bytes, pool, rb->main) != cudaSuccess)
        return -1;
    rb->arena_cap = bytes;
    return 0;
}

/* Validate, assign series to buckets, compute every offset and carve the buffers. */
static int plan(ssa_rbatch *rb, int B, const int *N, const int *L, const int *k)
{
    for (int s = 0; s < B; s++)
    {
        if (N[s] < 4 || L[s] < 2 || L[s] > N[s] - 1 || k[s] < 1)
            return -1;
        const int K = N[s] - L[s] + 1;
        const int kp = imin(k[s] + (rb->followup ? 0 : rb->p), imin(L[s], K));
        if (kp > SSA_MAX_KP)
            return -1;
        const int logh = ssad_fft_code_for(N[s]);
        if (logh >= RB_NB || logh < RB_MIN_LOGH || ssad_fft_h(logh) == 0)
            return -1;
    }
    int count[RB_NB] = {0};
    for (int s = 0; s < B; s++)
        count[bucket_of(ssad_fft_code_for(N[s]))]++;
    for (int g = 0; g < RB_NB; g++)
        if (count[g] > 65535) /* the job index is blockIdx.y in the column kernels */
            return -1;
    for (int g = 0; g < RB_NB; g++)
    {
        rbucket *b = &rb->bk[g];
        b->nb = 0;
        if (!count[g])
            continue;
        if (bucket_setup(b, g, rb->prof) != 0)
            return -1;
        b->multi = bucket_of(SSA_MULTI_MIN_LOGH) == g && g_multi;
        if (count[g] > b->cap_nb)
        {
            rser *sd = (rser *)realloc(b->sd, sizeof(rser) * count[g]);
            if (!sd)
                return -1;
            b->sd = sd;
            b->cap_nb = count[g];
        }
    }
    /* packed batch offsets */
    size_t ox = 0, osig = 0, oW = 0, ogrp = 0;
    for (int s = 0; s < B; s++)
    {
        const int code = ssad_fft_code_for(N[s]);
        rbucket *b = &rb->bk[bucket_of(code)];
        rser *S = &b->sd[b->nb++];
        memset(S, 0, sizeof(*S));
        S->src = s;
        S->code = code;
        S->ldS = round4(2LL * (ssad_fft_h(code) + 1) + 2);
        S->N = N[s];
        S->L = L[s];
        S->K = N[s] - L[s] + 1;
        S->kp = imin(k[s] + (rb->followup ? 0 : rb->p), imin(S->L, S->K));
        S->k = imin(k[s], S->kp);
        if (rb->followup)
        {
            S->Ux = rb->fu_U[s];
            S->Vx = rb->fu_V[s];
            S->sx = rb->fu_sig[s];
            S->gx = rb->d_fu_gidx + rb->fu_goff[s];
            S->gn = rb->fu_goff[s + 1] - rb->fu_goff[s];
            S->gmax = -1;
            for (int e = rb->fu_goff[s]; e < rb->fu_goff[s + 1]; e++)
                if (rb->h_fu_gidx[e] < S->k && rb->h_fu_gidx[e] > S->gmax)
                    S->gmax = rb->h_fu_gidx[e];
        }
        S->ox = ox;
        S->osig = osig;
        S->oW = oW;
        S->ogrp = ogrp;
        ox += (size_t)S->N;
        osig += (size_t)S->k;
        oW += (size_t)S->k * S->k;
        ogrp += (size_t)rb->n_groups * S->N;
        rb->h_off[4 * s + 0] = S->ox;
        rb->h_off[4 * s + 1] = S->osig;
        rb->h_off[4 * s + 2] = S->oW;
        rb->h_off[4 * s + 3] = S->ogrp;
    }
    rb->n_x = ox;
    rb->n_sig = osig;
    rb->n_W = oW;
    rb->n_grp = ogrp;
    /* per-bucket offsets and buffers */
    for (int g = 0; g < RB_NB; g++)
    {
        rbucket *b = &rb->bk[g];
        if (!b->nb)
            continue;
        size_t oY = 0, oZ = 0, opart = 0, oqsum = 0, oR = 0, oZu = 0, orecon = 0, onorm = 0, ospec = 0, oX = 0;
        for (int i = 0; i < b->nb; i++)
        {
            rser *S = &b->sd[i];
            S->ldL = round4(S->L);
            S->ldK = round4(S->K);
            S->ldN = round4(S->N);
            S->rows_L = gram_rows_for(S->L, b->nb, g);
            S->rows_K = gram_rows_for(S->K, b->nb, g);
            S->rows_N = imin(gram_rows_for(S->N, b->nb, g), SSA_W_MAX_ROWS);
            S->nch_L = (S->L + S->rows_L - 1) / S->rows_L;
            S->nch_K = (S->K + S->rows_K - 1) / S->rows_K;
            S->nch_N = (S->N + S->rows_N - 1) / S->rows_N;
            S->rows_W = ssad_wcorr_tc() ? imax(S->rows_N, SSA_TC_MIN_ROWS) : S->rows_N;
            S->nch_W = (S->N + S->rows_W - 1) / S->rows_W;
            S->nq = (S->L + SSA_ROWMUL_ROWS - 1) / SSA_ROWMUL_ROWS;
            S->wantW = !rb->followup && (!rb->cur_wmask || rb->cur_wmask[S->src]);
            S->nelem = rb->followup ? S->gmax + 1 : S->wantW ? S->k : imin(S->k, rb->grp_need);
            S->oY = oY;
            S->oZ = oZ;
            S->opart = opart;
            S->oqsum = oqsum;
            S->oR = oR;
            S->oZu = oZu;
            S->orecon = orecon;
            S->onorm = onorm;
            S->ospec = ospec;
            S->oX = oX;
            oX += (size_t)S->ldS;
            oY += (size_t)S->ldL * S->kp;
            oZ += (size_t)S->ldK * S->kp;
            opart += (size_t)imax(S->nch_L, imax(S->nch_K, S->nch_N)) * S->kp * (S->kp + 1) / 2;
            oqsum += (size_t)S->nq * S->kp;
            oR += (size_t)S->kp * S->kp;
            oZu += (size_t)S->kp * S->k;
            orecon += (size_t)S->nelem * S->ldN;
            onorm += (size_t)S->k;
            ospec += (size_t)S->nelem * S->ldS;
        }
        /* one run pushes 13 + 6 q job tables of at most sizeof(ssa_col_job) bytes per series,
         * each 16-byte aligned (a multi-length bucket pushes the per-code stages in up to six
         * parts), and per sweep a column list or tile table of at most SSA_MAX_KP entries per
         * series */
        size_t arena = ((size_t)b->nb * sizeof(ssa_col_job) + 16 * 6) * (size_t)(16 + 6 * rb->q) + (1 << 16);
        arena += (size_t)(2 * rb->q + 2) * ((size_t)SSA_MAX_KP * b->nb + 2) * sizeof(ssa_tile);
        const void *ja_old = b->e.ja.d;
        if (ssae_grow_arena(&b->e, arena) != 0)
            return -1;
        if (ja_old && b->e.ja.d != ja_old)
        {
            /* captured graphs copy from and read the old staging areas: drop them (the previous
             * run, graphs included, has completed: quiesce waited for it) */
            for (int i = 0; i < 4; i++)
                graph_free(&rb->graphs[i]);
            rb->last_sig = 0;
        }
        b->sz[0] = oX * sizeof(float); /* X */
        b->sz[1] = oY * sizeof(float);
        b->sz[2] = oZ * sizeof(float);
        b->sz[3] = opart * sizeof(double);
        b->sz[4] = oqsum * sizeof(double);
        b->sz[5] = oR * sizeof(double);
        b->sz[6] = oZu * sizeof(float);
        b->sz[7] = oZu * sizeof(float);
        b->sz[8] = orecon * sizeof(float);
        b->sz[9] = onorm * sizeof(double);
        b->sz[10] = b->logh > SSA_ELEM2_MAX_LOGH ? ospec * sizeof(float) : 0;
        if (rb->followup) /* no decomposition: no signal spectra, probe blocks, Grams or rotations */
            for (int i = 0; i < 8; i++)
                b->sz[i] = 0;
    }
    /* carve the arena: every bucket's buffers, then the packed outputs and status words */
    size_t need = 0;
    for (int g = 0; g < RB_NB; g++)
        if (rb->bk[g].nb)
            for (int i = 0; i < 11; i++)
                need += (rb->bk[g].sz[i] + 255) & ~(size_t)255;
    if (rb->followup)
        rb->n_sig = rb->n_W = 0;
    const size_t tail[5] = {rb->n_sig * sizeof(double), rb->n_W * sizeof(double),
                            rb->n_groups > 0 ? rb->n_grp * sizeof(double) : 0, (size_t)B * sizeof(int),
                            (size_t)B * sizeof(int)};
    for (int i = 0; i < 5; i++)
        need += (tail[i] + 255) & ~(size_t)255;
    if (need > rb->arena_cap && ssa_rbatch_reserve(rb, need + need / 8) != 0)
        return -1;
    size_t off = 0;
#define RB_CARVE(ptr, bytes)                                  \
    do                                                        \
    {                                                         \
        (ptr) = (void *)(rb->arena + off);                    \
        off += ((size_t)(bytes) + 255) & ~(size_t)255;        \
    } while (0)
    for (int g = 0; g < RB_NB; g++)
    {
        rbucket *b = &rb->bk[g];
        if (!b->nb)
            continue;
        void *v;
        RB_CARVE(v, b->sz[0]);
        b->X = (float *)v;
        RB_CARVE(v, b->sz[1]);
        b->Y = (float *)v;
        RB_CARVE(v, b->sz[2]);
        b->Z = (float *)v;
        RB_CARVE(v, b->sz[3]);
        b->part = (double *)v;
        RB_CARVE(v, b->sz[4]);
        b->qsum = (double *)v;
        RB_CARVE(v, b->sz[5]);
        b->R = (double *)v;
        RB_CARVE(v, b->sz[6]);
        b->Zu = (float *)v;
        RB_CARVE(v, b->sz[7]);
        b->Zv = (float *)v;
        RB_CARVE(v, b->sz[8]);
        b->recon = (float *)v;
        RB_CARVE(v, b->sz[9]);
        b->norm2 = (double *)v;
        RB_CARVE(v, b->sz[10]);
        b->Us = b->sz[10] ? (float *)v : NULL;
    }
    {
        void *v;
        RB_CARVE(v, tail[0]);
        rb->sigma = (double *)v;
        RB_CARVE(v, tail[1]);
        rb->W = (double *)v;
        RB_CARVE(v, tail[2]);
        rb->groups = rb->n_groups > 0 ? (double *)v : NULL;
        RB_CARVE(v, tail[3]);
        rb->status = (int *)v;
        RB_CARVE(v, tail[4]);
        rb->lrf_status = (int *)v;
    }
#undef RB_CARVE
    return 0;
}

/* ---- entry points ------------------------------------------------------------------------ */

/* Wait for the previous run on every stream and reset the job arenas. */
/* Before a run reuses the buckets' host job tables: the previous run's bucket streams have
 * consumed them. The main stream is not waited for: it may already hold this run's inputs, and
 * the new run's buckets are ordered after it anyway. */
static int quiesce(ssa_rbatch *rb)
{
    int rc = 0;
    if (rb->graph_pending)
    {
        /* the graph's copy nodes read the staging areas and the seeds when they execute */
        rc |= cudaEventSynchronize(rb->ev_graph) != cudaSuccess;
        rb->graph_pending = 0;
    }
    for (int g = 0; g < RB_NB; g++)
        if (rb->bk[g].live)
        {
            rc |= cudaStreamSynchronize(rb->bk[g].e.st) != cudaSuccess;
            ssae_reset_jobs(&rb->bk[g].e);
        }
    return rc ? -1 : 0;
}

static int ensure_hoff(ssa_rbatch *rb, int B)
{
    size_t *h = (size_t *)realloc(rb->h_off, sizeof(size_t) * 4 * (size_t)B);
    if (!h)
        return -1;
    rb->h_off = h;
    return 0;
}

/* The work of a run after plan(): seeds, output clears, every bucket's pipeline on its stream,
 * joined back into the main stream. */
static int enqueue_body(ssa_rbatch *rb, int B, const double *d_x, unsigned long long seed)
{
    if (!rb->followup &&
        cudaMemcpyAsync(rb->d_seeds, rb->h_seeds, sizeof(unsigned long long) * B, cudaMemcpyHostToDevice, rb->main) !=
            cudaSuccess)
        return -1;
    if (rb->cur_wmask && rb->n_W > 0 &&
        cudaMemsetAsync(rb->W, 0, sizeof(double) * rb->n_W, rb->main) != cudaSuccess)
        return -1;
    if (cudaMemsetAsync(rb->status, 0, sizeof(int) * B, rb->main) != cudaSuccess ||
        cudaMemsetAsync(rb->lrf_status, 0, sizeof(int) * B, rb->main) != cudaSuccess ||
        cudaEventRecord(rb->ev_in, rb->main) != cudaSuccess)
        return -1;
    /* largest FFT lengths first: they take longest. Profiling mode 2 chains the buckets (each
     * waits for the previous one) so that every launch's event interval is its own. */
    cudaEvent_t prev = rb->ev_in;
    for (int g = RB_NB - 1; g >= 0; g--)
    {
        rbucket *b = &rb->bk[g];
        if (!b->nb)
            continue;
        b->status_base = rb->status;
        if (cudaStreamWaitEvent(b->e.st, rb->prof == 2 ? prev : rb->ev_in, 0) != cudaSuccess ||
            (rb->followup ? bucket_followup(b, rb) : bucket_run(b, rb, d_x, seed)) != 0 ||
            cudaEventRecord(b->done, b->e.st) != cudaSuccess ||
            cudaStreamWaitEvent(rb->main, b->done, 0) != cudaSuccess)
            return -1;
        prev = b->done;
    }
    return 0;
}

/* FNV-1a over the bytes of everything a captured run bakes in: shapes, per-series options,
 * device addresses (input, arena, job tables, seeds) and the global switches. */
static unsigned long long fnv(unsigned long long h, const void *p, size_t n)
{
    const unsigned char *c = (const unsigned char *)p;
    for (size_t i = 0; i < n; i++)
        h = (h ^ c[i]) * 0x100000001B3ull;
    return h;
}

static unsigned long long run_signature(const ssa_rbatch *rb, int B, const int *N, const int *L, const int *k,
                                        const double *d_x)
{
    unsigned long long h = 0xCBF29CE484222325ull;
    const int head[10] = {B, rb->p, rb->q, rb->n_groups, rb->lrf_slot, rb->n_lrf_group, g_multi, ssad_wcorr_tc(),
                          ssad_cl14(), ssad_rowmul_tc_on()};
    h = fnv(h, head, sizeof(head));
    h = fnv(h, N, sizeof(int) * B);
    h = fnv(h, L, sizeof(int) * B);
    h = fnv(h, k, sizeof(int) * B);
    const void *ptrs[4] = {d_x, rb->arena, rb->d_seeds, rb->d_lrf_group};
    h = fnv(h, ptrs, sizeof(ptrs));
    for (int s = 0; s < B; s++)
    {
        const unsigned char w = rb->cur_wmask ? rb->cur_wmask[s] : 1;
        const void *lp = rb->cur_lrf ? (const void *)rb->cur_lrf[s] : NULL;
        h = fnv(h, &w, 1);
        h = fnv(h, &lp, sizeof(lp));
    }
    for (int g = 0; g < RB_NB; g++)
        if (rb->bk[g].nb)
        {
            const void *jd = rb->bk[g].e.ja.d;
            h = fnv(h, &g, sizeof(g));
            h = fnv(h, &jd, sizeof(jd));
        }
    return h;
}

static void graph_free(struct rgraph *g)
{
    if (g->exec)
        cudaGraphExecDestroy(g->exec);
    for (int i = 0; i < RB_NB; i++)
        free(g->snap[i]);
    memset(g, 0, sizeof(*g));
}

/* replay != 0: the graph's kernels join the launch count (a capture counted them already). */
static int graph_launch(ssa_rbatch *rb, struct rgraph *g, int replay)
{
    g->stamp = ++rb->gstamp;
    if (replay)
        ssad_count_launches(g->kernels);
    if (cudaGraphLaunch(g->exec, rb->main) != cudaSuccess || cudaEventRecord(rb->ev_graph, rb->main) != cudaSuccess)
        return -1;
    rb->graph_pending = 1;
    return 0;
}

/* Enqueue a run whose packed input d_x is ready at the main stream's current position. */
static int run_enqueue(ssa_rbatch *rb, int B, const int *N, const int *L, const int *k, const double *d_x,
                       unsigned long long seed)
{
    if (ensure_hoff(rb, B) != 0 || plan(rb, B, N, L, k) != 0)
        return -1;
    rb->B = B;
    if (!rb->followup)
    {
        if ((size_t)B > rb->c_seeds)
        {
            if (rb->h_seeds)
                cudaFreeHost(rb->h_seeds);
            if (rb->d_seeds)
                cudaFree(rb->d_seeds);
            rb->h_seeds = NULL;
            rb->d_seeds = NULL;
            rb->c_seeds = 0;
            const size_t c = (size_t)B + (size_t)B / 2 + 64;
            if (cudaMallocHost((void **)&rb->h_seeds, sizeof(unsigned long long) * c) != cudaSuccess ||
                cudaMalloc((void **)&rb->d_seeds, sizeof(unsigned long long) * c) != cudaSuccess)
                return -1;
            rb->c_seeds = c;
        }
        for (int s = 0; s < B; s++)
            rb->h_seeds[s] = rb->cur_seeds ? rb->cur_seeds[s]
                                           : seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(s + 1));
    }
    const int use = rb->graphs_on && !rb->prof && !rb->followup;
    const unsigned long long sig = use ? run_signature(rb, B, N, L, k, d_x) : 0;
    if (use)
        for (int i = 0; i < 4; i++)
        {
            struct rgraph *g = &rb->graphs[i];
            if (!g->exec || g->sig != sig)
                continue;
            /* replay: the job tables of the captured run back into the staging areas */
            for (int b = 0; b < RB_NB; b++)
                if (g->snap_n[b])
                {
                    memcpy(rb->bk[b].e.ja.h, g->snap[b], g->snap_n[b]);
                    rb->bk[b].e.ja.used = g->snap_n[b];
                }
            rb->n_replays++;
            return graph_launch(rb, g, 1);
        }
    const int capture = use && sig == rb->last_sig;
    rb->last_sig = sig;
    if (!capture)
        return enqueue_body(rb, B, d_x, seed);
    if (cudaStreamBeginCapture(rb->main, cudaStreamCaptureModeRelaxed) != cudaSuccess)
        return -1;
    const unsigned long long k0 = ssad_launch_count();
    const int rc = enqueue_body(rb, B, d_x, seed);
    const unsigned long long nk = ssad_launch_count() - k0;
    cudaGraph_t graph = NULL;
    const cudaError_t ec = cudaStreamEndCapture(rb->main, &graph);
    cudaGraphExec_t exec = NULL;
    if (rc != 0 || ec != cudaSuccess || !graph || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
    {
        if (graph)
            cudaGraphDestroy(graph);
        cudaGetLastError();
        /* nothing of the captured work ran: run it directly, and leave graphs off for this batch */
        rb->graphs_on = 0;
        for (int b = 0; b < RB_NB; b++)
            rb->bk[b].e.ja.used = 0;
        return enqueue_body(rb, B, d_x, seed);
    }
    cudaGraphDestroy(graph);
    int slot = 0;
    for (int i = 1; i < 4; i++)
        if (rb->graphs[i].stamp < rb->graphs[slot].stamp)
            slot = i;
    struct rgraph *g = &rb->graphs[slot];
    graph_free(g);
    g->sig = sig;
    g->exec = exec;
    g->kernels = nk;
    for (int b = 0; b < RB_NB; b++)
    {
        const size_t n = rb->bk[b].nb ? rb->bk[b].e.ja.used : 0;
        if (n && (g->snap[b] = (char *)malloc(n)) != NULL)
        {
            memcpy(g->snap[b], rb->bk[b].e.ja.h, n);
            g->snap_n[b] = n;
        }
        else if (n)
        {
            graph_free(g);
            return -1;
        }
    }
    rb->n_captures++;
    return graph_launch(rb, g, 0);
}

int ssa_rbatch_set_graphs(ssa_rbatch *rb, int on)
{
    if (!rb)
        return -1;
    rb->graphs_on = on != 0;
    return 0;
}

int ssa_rbatch_graph_stats(const ssa_rbatch *rb, long long *captures, long long *replays)
{
    if (!rb)
        return -1;
    if (captures)
        *captures = rb->n_captures;
    if (replays)
        *replays = rb->n_replays;
    return 0;
}

int ssa_rbatch_run_device(ssa_rbatch *rb, int B, const int *N, const int *L, const int *k, const double *d_x,
                          uint64_t seed)
{
    return ssa_rbatch_run_device_ex(rb, B, N, L, k, d_x, seed, NULL);
}

int ssa_rbatch_run_device_ex(ssa_rbatch *rb, int B, const int *N, const int *L, const int *k, const double *d_x,
                             uint64_t seed, const unsigned char *want_w)
{
    if (!rb || B < 1 || !N || !L || !k || !d_x)
        return -1;
    if (quiesce(rb) != 0)
        return -1;
    rb->cur_wmask = want_w;
    const int rc = run_enqueue(rb, B, N, L, k, d_x, (unsigned long long)seed);
    rb->cur_wmask = NULL;
    return rc;
}

int ssa_rbatch_sync(ssa_rbatch *rb)
{
    if (!rb)
        return -1;
    if (cudaStreamSynchronize(rb->main) != cudaSuccess)
        return -1;
    if (rb->B <= 0)
        return 0;
    int *st = (int *)malloc(sizeof(int) * rb->B);
    if (!st)
        return -1;
    int rc = cudaMemcpy(st, rb->status, sizeof(int) * rb->B, cudaMemcpyDeviceToHost) != cudaSuccess;
    for (int s = 0; s < rb->B && !rc; s++)
        if (st[s] != 0)
            rc = 1;
    free(st);
    return rc ? -1 : 0;
}

int ssa_rbatch_run(ssa_rbatch *rb, int B, const int *N, const int *L, const int *k, const double *x, uint64_t seed,
                   double *sigma, double *W, double *groups)
{
    return ssa_rbatch_run_ex(rb, B, N, L, k, x, seed, sigma, W, groups, NULL);
}

int ssa_rbatch_run_ex(ssa_rbatch *rb, int B, const int *N, const int *L, const int *k, const double *x, uint64_t seed,
                      double *sigma, double *W, double *groups, const unsigned char *want_w)
{
    if (!rb || B < 1 || !N || !L || !k || !x)
        return -1;
    size_t nx = 0;
    for (int s = 0; s < B; s++)
    {
        if (N[s] < 1)
            return -1;
        nx += (size_t)N[s];
    }
    if (quiesce(rb) != 0 || grow((void **)&rb->d_xs, &rb->c_xs, nx, sizeof(double), rb->main) != 0)
        return -1;
    if (cudaMemcpyAsync(rb->d_xs, x, sizeof(double) * nx, cudaMemcpyHostToDevice, rb->main) != cudaSuccess)
        return -1;
    rb->cur_wmask = want_w;
    const int rq = run_enqueue(rb, B, N, L, k, rb->d_xs, (unsigned long long)seed);
    rb->cur_wmask = NULL;
    if (rq != 0)
        return -1;
    if (sigma && cudaMemcpyAsync(sigma, rb->sigma, sizeof(double) * rb->n_sig, cudaMemcpyDeviceToHost, rb->main) !=
                     cudaSuccess)
        return -1;
    if (W && cudaMemcpyAsync(W, rb->W, sizeof(double) * rb->n_W, cudaMemcpyDeviceToHost, rb->main) != cudaSuccess)
        return -1;
    if (groups && rb->n_groups > 0 &&
        cudaMemcpyAsync(groups, rb->groups, sizeof(double) * rb->n_grp, cudaMemcpyDeviceToHost, rb->main) !=
            cudaSuccess)
        return -1;
    return ssa_rbatch_sync(rb);
}

int ssa_rbatch_layout(const ssa_rbatch *rb, size_t *offsets, size_t *totals)
{
    if (!rb || rb->B <= 0)
        return -1;
    if (offsets)
        memcpy(offsets, rb->h_off, sizeof(size_t) * 4 * (size_t)rb->B);
    if (totals)
    {
        totals[0] = rb->n_x;
        totals[1] = rb->n_sig;
        totals[2] = rb->n_W;
        totals[3] = rb->n_grp;
    }
    return rb->B;
}

/* Series s of the last run: its bucket entry, or NULL. */
static const rser *find_series(const ssa_rbatch *rb, int s, const rbucket **bk)
{
    for (int g = 0; g < RB_NB; g++)
    {
        const rbucket *b = &rb->bk[g];
        for (int i = 0; i < b->nb; i++)
            if (b->sd[i].src == s)
            {
                *bk = b;
                return &b->sd[i];
            }
    }
    return NULL;
}

static int copy_cols_f32(double *dst, const float *src, long long ld, int m, int n, float *tmp)
{
    if (cudaMemcpy2D(tmp, sizeof(float) * (size_t)m, src, sizeof(float) * (size_t)ld, sizeof(float) * (size_t)m,
                     (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    for (size_t i = 0; i < (size_t)m * n; i++)
        dst[i] = (double)tmp[i];
    return 0;
}

int ssa_rbatch_series_result(ssa_rbatch *rb, int s, double *sigma, double *W, double *groups, double *U, double *V)
{
    if (!rb || s < 0 || s >= rb->B)
        return -1;
    const rbucket *b = NULL;
    const rser *S = find_series(rb, s, &b);
    if (!S || cudaStreamSynchronize(rb->main) != cudaSuccess)
        return -1;
    const int k = S->k;
    if (sigma && cudaMemcpy(sigma, rb->sigma + S->osig, sizeof(double) * (size_t)k, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    if (W && cudaMemcpy(W, rb->W + S->oW, sizeof(double) * (size_t)k * k, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    if (groups && rb->n_groups > 0 &&
        cudaMemcpy(groups, rb->groups + S->ogrp, sizeof(double) * (size_t)rb->n_groups * S->N,
                   cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    if (U || V)
    {
        float *tmp = (float *)malloc(sizeof(float) * (size_t)imax(S->L, S->K) * k);
        if (!tmp)
            return -1;
        int rc = 0;
        if (U)
            rc |= copy_cols_f32(U, b->Y + S->oY, S->ldL, S->L, k, tmp);
        if (V)
            rc |= copy_cols_f32(V, b->Z + S->oZ, S->ldK, S->K, k, tmp);
        free(tmp);
        if (rc)
            return -1;
    }
    return k;
}

int ssa_rbatch_device_results(const ssa_rbatch *rb, ssa_batch_results *out)
{
    if (!rb || !out)
        return -1;
    memset(out, 0, sizeof(*out));
    out->sigma = rb->sigma;
    out->W = rb->W;
    out->groups = rb->groups;
    out->status = rb->status;
    out->stream = (void *)rb->main;
    return 0;
}

int ssa_rbatch_set_profiling(ssa_rbatch *rb, int on)
{
    if (!rb || on < 0 || on > 2)
        return -1;
    rb->prof = on;
    for (int g = 0; g < RB_NB; g++)
        if (rb->bk[g].live && ssae_set_profiling(&rb->bk[g].e, on) != 0)
            return -1;
    return 0;
}

/* Stage times summed over the buckets (buckets overlap on the device, so the sum can exceed the
 * wall time of a run). */
int ssa_rbatch_profile(ssa_rbatch *rb, double *ms, long long *launches, int nkinds)
{
    if (!rb || !ms || !launches)
        return -1;
    const int n = nkinds < SSAK_NKINDS ? nkinds : SSAK_NKINDS;
    for (int k = 0; k < n; k++)
    {
        ms[k] = 0.0;
        launches[k] = 0;
    }
    for (int g = 0; g < RB_NB; g++)
    {
        rbucket *b = &rb->bk[g];
        if (!b->live)
            continue;
        if (ssae_prof_collect(&b->e) != 0)
            return -1;
        for (int k = 0; k < n; k++)
        {
            ms[k] += b->e.prof_ms[k];
            launches[k] += b->e.prof_n[k];
        }
        for (int k = 0; k < SSAK_NKINDS; k++)
        {
            b->e.prof_ms[k] = 0.0;
            b->e.prof_n[k] = 0;
        }
    }
    return SSAK_NKINDS;
}

/* ---- extensions for the request server (ssa_ragged_int.h) ------------------------------- */

int ssar_set_lrf_group(ssa_rbatch *rb, int slot, const int *group, int n_group)
{
    if (!rb || slot < 0 || slot >= rb->n_groups || n_group < 1 || n_group > SSA_MAX_KP)
        return -1;
    int gmax = 0;
    for (int i = 0; i < n_group; i++)
    {
        if (group[i] < 0 || group[i] >= SSA_MAX_KP)
            return -1;
        gmax = imax(gmax, group[i]);
    }
    if (!rb->d_lrf_group && cudaMalloc((void **)&rb->d_lrf_group, sizeof(int) * SSA_MAX_KP) != cudaSuccess)
        return -1;
    if (cudaMemcpy(rb->d_lrf_group, group, sizeof(int) * n_group, cudaMemcpyHostToDevice) != cudaSuccess)
        return -1;
    rb->lrf_slot = slot;
    rb->n_lrf_group = n_group;
    rb->lrf_gmax = gmax;
    return 0;
}

int ssar_run_enqueue_ex(ssa_rbatch *rb, int B, const int *N, const int *L, const int *k, const double *d_x,
                        const unsigned long long *seeds, double *const *lrf_dst, const unsigned char *want_w)
{
    if (!rb || B < 1 || !N || !L || !k || !d_x)
        return -1;
    static int trace = -1;
    if (trace < 0)
    {
        const char *ev = getenv("SSA_SERVER_TRACE");
        trace = ev && ev[0] == '1';
    }
    struct timespec q0, q1;
    clock_gettime(CLOCK_MONOTONIC, &q0);
    if (quiesce(rb) != 0)
        return -1;
    clock_gettime(CLOCK_MONOTONIC, &q1);
    const double qms = 1e3 * (double)(q1.tv_sec - q0.tv_sec) + 1e-6 * (double)(q1.tv_nsec - q0.tv_nsec);
    if (trace && qms > 2.0)
        fprintf(stderr, "ssa_rbatch: waited %.1f ms for the previous run before enqueueing\n", qms);
    rb->cur_seeds = seeds;
    rb->cur_lrf = lrf_dst;
    rb->cur_wmask = want_w;
    int rc = run_enqueue(rb, B, N, L, k, d_x, 0);
    rb->cur_seeds = NULL;
    rb->cur_lrf = NULL;
    rb->cur_wmask = NULL;
    return rc;
}

int ssar_run_followup(ssa_rbatch *rb, int B, const int *N, const int *L, const int *k, const float *const *U,
                      const float *const *V, const double *const *sig, const int *gidx, const int *goff,
                      double *const *lrf_dst)
{
    if (!rb || B < 1 || !N || !L || !k || !U || !V || !sig || !gidx || !goff || rb->n_groups < 1)
        return -1;
    if (quiesce(rb) != 0)
        return -1;
    /* every series' group, uploaded on the main stream ahead of the buckets (which wait for it) */
    const size_t ng = (size_t)goff[B];
    if (ng + 1 > rb->c_fu_gidx)
    {
        if (rb->h_fu_gidx)
            cudaFreeHost(rb->h_fu_gidx);
        if (rb->d_fu_gidx)
            cudaFree(rb->d_fu_gidx);
        rb->h_fu_gidx = NULL;
        rb->d_fu_gidx = NULL;
        rb->c_fu_gidx = 0;
        const size_t c = ng + ng / 2 + 64;
        if (cudaMallocHost((void **)&rb->h_fu_gidx, sizeof(int) * c) != cudaSuccess ||
            cudaMalloc((void **)&rb->d_fu_gidx, sizeof(int) * c) != cudaSuccess)
            return -1;
        rb->c_fu_gidx = c;
    }
    else if (cudaStreamSynchronize(rb->main) != cudaSuccess) /* the previous run's upload is done */
        return -1;
    memcpy(rb->h_fu_gidx, gidx, sizeof(int) * ng);
    if (cudaMemcpyAsync(rb->d_fu_gidx, rb->h_fu_gidx, sizeof(int) * ng, cudaMemcpyHostToDevice, rb->main) !=
        cudaSuccess)
        return -1;
    rb->followup = 1;
    rb->fu_U = U;
    rb->fu_V = V;
    rb->fu_sig = sig;
    rb->fu_goff = goff;
    rb->cur_lrf = lrf_dst;
    /* d_x is not read by a follow-up run: any valid pointer */
    int rc = run_enqueue(rb, B, N, L, k, (const double *)rb->d_fu_gidx, 0);
    rb->followup = 0;
    rb->fu_U = rb->fu_V = NULL;
    rb->fu_sig = NULL;
    rb->fu_goff = NULL;
    rb->cur_lrf = NULL;
    return rc;
}

int ssar_series_factors(const ssa_rbatch *rb, int s, const float **U, const float **V)
{
    const rbucket *b = NULL;
    const rser *S = find_series(rb, s, &b);
    if (!S)
        return -1;
    *U = b->Y + S->oY;
    *V = b->Z + S->oZ;
    return S->k;
}

cudaStream_t ssar_main_stream(const ssa_rbatch *rb) { return rb->main; }
const int *ssar_status(const ssa_rbatch *rb) { return rb->status; }
const int *ssar_lrf_status(const ssa_rbatch *rb) { return rb->lrf_status; }
const double *ssar_sigma(const ssa_rbatch *rb) { return rb->sigma; }
const double *ssar_W(const ssa_rbatch *rb) { return rb->W; }
const double *ssar_groups(const ssa_rbatch *rb) { return rb->groups; }
const size_t *ssar_offsets(const ssa_rbatch *rb) { return rb->h_off; }
void ssar_totals(const ssa_rbatch *rb, size_t *t4)
{
    t4[0] = rb->n_x;
    t4[1] = rb->n_sig;
    t4[2] = rb->n_W;
    t4[3] = rb->n_grp;
}

/* Device bytes one series of this shape occupies in a bucket and in the packed outputs. */
size_t ssar_series_bytes(int N, int L, int k, int p, int n_groups)
{
    const int K = N - L + 1;
    const int kp = imin(k + p, imin(L, K));
    k = imin(k, kp);
    const int logh = ssad_fft_code_for(N);
    const size_t ldS = (size_t)round4(2LL * (ssad_fft_h(logh) + 1) + 2);
    const int nb_est = 64; /* Gram chunking at moderate bucket sizes */
    const int nch = imax(imax((L + gram_rows(L, nb_est) - 1) / gram_rows(L, nb_est),
                              (K + gram_rows(K, nb_est) - 1) / gram_rows(K, nb_est)),
                         (N + imin(gram_rows(N, nb_est), SSA_W_MAX_ROWS) - 1) /
                             imin(gram_rows(N, nb_est), SSA_W_MAX_ROWS));
    size_t b = 0;
    b += 4 * ldS;                                               /* X */
    b += 4 * (size_t)(round4(L) + round4(K)) * kp;               /* Y, Z */
    b += 8 * (size_t)nch * kp * (kp + 1) / 2;                    /* part */
    b += 8 * (size_t)((L + SSA_ROWMUL_ROWS - 1) / SSA_ROWMUL_ROWS) * kp; /* qsum */
    b += 8 * (size_t)kp * kp + 8 * (size_t)kp * k;               /* R^{-1} (FP64), Zu, Zv */
    b += 4 * (size_t)k * round4(N) + 8 * (size_t)k;              /* recon, norm2 */
    if (logh > SSA_ELEM2_MAX_LOGH)
        b += 4 * (size_t)k * ldS;                                /* Us */
    b += 8 * ((size_t)N + k + (size_t)k * k + (size_t)n_groups * N); /* x, sigma, W, groups */
    return b + b / 8;                                           /* growth slack */
}
