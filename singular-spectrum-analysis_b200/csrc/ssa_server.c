/*
 * Request server: continuous batching of decompose / reconstruct / W-correlation / forecast
 * requests of mixed size on one GPU.
 *
 * One worker thread owns the device work. Requests are queued by ssa_server_submit (any thread)
 * and taken in arrival order. Decompositions are gathered into uneven batches (ssa_ragged.c),
 * each batch bounded by a device-memory share of the HBM budget; up to `max_inflight` batches
 * run at once on their own streams, so requests that arrive while others are on the GPU start
 * as soon as a batch slot is free and overlap with the running ones. A batch is ordered by
 * FFT-length bucket, and each bucket's requests complete when that bucket's part of the run and
 * its output copies are done, ahead of the batch's longer buckets. A decomposition request
 * leaves its series resident: its factors U, V, sigma, its signal, the LRF coefficients of the
 * forecast group [0, 1, 2] and the last L - 1 values of that group's reconstruction stay in
 * device memory (stream-ordered pool, least recently used entries evicted beyond the resident
 * share of the budget). Follow-ups on a resident series do not decompose again: a default
 * forecast runs the recurrence only (batched, one CTA per request); reconstructions and forecasts
 * of caller-chosen groups run as follow-up batches (elementary reconstructions of the resident
 * factors, group sums, LRF, recurrence); Cadzow requests run on a worker of their own, a resident
 * series' first projection taken from its factors. Every request is stamped with its arrival and
 * completion times on the host's monotonic clock; completion means its outputs are in host
 * memory.
 */
#include <errno.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <cuda_runtime_api.h>

#include "ssa_engine.h"
#include "ssa_ragged_int.h"
#include "../../include/ssa_opt.h"

#define SRV_GROUPS 3 /* [0], [1, 2], [0, 1, 2] (forecast group) */

static const int g_group_idx[] = {0, 1, 2, 0, 1, 2};
static const int g_group_sizes[] = {1, 2, 3};
static const int g_fc_group[] = {0, 1, 2};
static int g_not_resident; /* marker: the request was seen and gets no resident entry */

enum
{
    RES_PENDING = 0,
    RES_READY = 1,
    RES_FAILED = 2
};

typedef struct res_entry
{
    int id;
    int state;
    int L;
    int refs;          /* in-flight follow-ups using it */
    int N, K, k;       /* shape and resident components */
    int lrf_ok;        /* the default forecast group's LRF is valid */
    long long ldL, ldK;
    /* one device block: doubles R (L-1), tail (L-1), verticality, sigma (k), signal (N), then
     * floats U (ldL x k) and V (ldK x k), the leading dimensions of the batch's factor blocks */
    double *d;
    double *sig, *x;
    float *U, *V;
    size_t bytes;
    size_t aoff; /* offset in the resident arena, or SIZE_MAX when from the pool */
    struct res_entry *prev, *next; /* LRU list, most recent first */
    struct res_entry *hnext;
} res_entry;

typedef struct
{
    ssa_rbatch *rb;
    int busy;
    int n, cap;
    ssa_request **req;
    int *N, *L, *k;
    unsigned long long *seeds;
    double **lrf_dst;
    unsigned char *wantw; /* 1: the request asked for the W-correlation */
    res_entry **res;
    /* per request: offsets (doubles) of its input in d_x and, for pageable buffers, in the
     * pinned staging areas (SIZE_MAX = copied directly from / to the caller's pinned memory) */
    size_t *xoff, *sin, *sout;
    /* per request, device addresses of its page-locked caller buffers: input, sigma, groups, W
     * (NULL where staged or not asked for) */
    double **hp;
    double *h_in, *h_out; /* pinned staging, fixed at creation */
    double *h_in_d, *h_out_d; /* their device addresses */
    int *h_st, *h_lst;        /* max_batch status words */
    /* copy segments of the batch's input gather and output scatter (page-locked, read by the
     * copy kernel through its device address) */
    ssa_copy_seg *h_seg, *h_seg_d;
    size_t c_seg;
    double *d_x;
    size_t c_dx;
    size_t bytes, in_used, out_used;
    cudaEvent_t done;
    /* per-bucket completion: the batch is ordered by FFT-length bucket; range r holds requests
     * rlo[r] .. rhi[r] - 1 of one bucket, whose outputs and status words are copied on that
     * bucket's stream and which complete when rev[r] has fired, ahead of the rest of the batch */
    int nrange;
    int rlo[SSAR_NB], rhi[SSAR_NB], rdone[SSAR_NB];
    cudaEvent_t rev[SSAR_NB];
} slot_t;

typedef struct
{
    cudaStream_t st;
    cudaEvent_t done;
    int busy;
    int n, cap;
    ssa_request **req;
    res_entry **res;
    ssa_fc_job *h_jobs, *d_jobs;
    double *h_out, *d_out;
    size_t c_hout, c_dout;
} fslot_t;

/* Follow-up batch on resident factors: reconstructions, forecasts of caller-chosen groups and the
 * first projection of Cadzow requests on resident series. */
typedef struct
{
    ssa_rbatch *rb; /* created with one group slot; every series brings its own group */
    cudaEvent_t done;
    int busy, n, cap;
    ssa_request **req;
    res_entry **res;
    int *N, *L, *k, *goff, *gidx;
    int cgidx;
    const float **U, **V;
    const double **sig;
    double **lrf;
    size_t *tmpoff, *hoff;
    double *d_tmp; /* per group forecast: R (L-1), tail (L-1), verticality */
    size_t c_tmp;
    ssa_fc_job *h_fc, *d_fc;
    int c_fc;
    double *d_fcout;
    size_t c_fcout;
    double *h_out; /* pinned: reconstructions, resident signals (Cadzow), forecasts */
    size_t c_hout;
    int *h_lst;
} uslot_t;

/* Cadzow requests waiting for the Cadzow worker, with host copies of a resident series' signal
 * and first projection (NULL for requests that bring their own signal). */
typedef struct cz_item
{
    ssa_request *r;
    double *x, *y1;
    struct cz_item *next;
} cz_item;

struct ssa_server
{
    pthread_t th;
    int th_live;
    pthread_mutex_t mu;
    pthread_cond_t cv;      /* worker wake-up */
    pthread_cond_t cv_done; /* drain */
    int stop;
    /* submitted, not yet taken by the worker (ring) */
    ssa_request **q;
    int qhead, qcount, qcap;
    long long outstanding; /* submitted and not completed */
    /* worker-private */
    ssa_request **pend; /* taken, waiting for a slot (decompositions) or a target (forecasts) */
    int npend, cpend;
    slot_t *slots;
    int nslots;
    fslot_t fs;
    int p, q_iters, max_batch;
    size_t budget, batch_budget, res_budget, res_bytes;
    res_entry **htab;
    int hcap;
    res_entry *lru_head, *lru_tail;
    cudaStream_t pool_st;
    cudaEvent_t ev_pool;
    int device;
    ssa_server_stats stats;
    uslot_t us;
    /* resident arena (explicit budget): one device allocation of res_budget bytes, entries carved
     * first-fit from a sorted list of free spans (no driver call per entry) */
    char *res_arena;
    struct rspan
    {
        size_t off, len;
    } *spans;
    int nspans, cspans;
    /* Cadzow worker: its own thread, queue and wake-up */
    pthread_t cz_th;
    int cz_live, cz_stop;
    cz_item *cz_head, *cz_tail;
    pthread_cond_t cz_cv;
};

double ssa_server_now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static int imin(int a, int b) { return a < b ? a : b; }

/* Pinned staging per batch slot for callers' pageable buffers (allocated once at creation; a
 * batch admits pageable requests while their bytes fit). Page-locked caller buffers
 * (ssa_host_alloc or any cudaHostAlloc / cudaHostRegister memory) are copied directly. */
#define SRV_STAGE_IN (256u << 20)
#define SRV_STAGE_OUT (512u << 20)
#define SRV_DIRECT ((size_t)-1)

/* Segments of at most this many doubles: one CTA of the copy kernel each. */
#define SRV_SEG_CHUNK ((size_t)16384)

/* Device address of page-locked host memory; NULL for pageable memory (staged instead). */
static double *mapped(const void *p)
{
    if (!p)
        return NULL;
    struct cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        cudaGetLastError();
        return NULL;
    }
    return a.type == cudaMemoryTypeHost ? (double *)a.devicePointer : NULL;
}

static size_t seg_count(size_t n) { return (n + SRV_SEG_CHUNK - 1) / SRV_SEG_CHUNK; }

static int req_kout(const ssa_server *s, const ssa_request *r)
{
    const int K = r->N - r->L + 1;
    const int kp = imin(r->k + s->p, imin(r->L, K));
    return imin(r->k, kp);
}

/* Output bytes a decomposition request asks for (sigma, groups or W). */
static size_t req_out_doubles(const ssa_server *s, const ssa_request *r)
{
    const size_t ke = (size_t)req_kout(s, r);
    size_t n = r->sigma ? ke : 0;
    if (r->type == SSA_REQ_DECOMPOSE_RECON && r->groups)
        n += 2 * (size_t)r->N;
    if (r->type == SSA_REQ_DECOMPOSE_WCORR && r->W)
        n += ke * ke;
    return n;
}

/* Segments of the copy kernel for the input and the outputs of one request. */
static size_t req_segs(const ssa_server *s, const ssa_request *r)
{
    const size_t ke = (size_t)req_kout(s, r);
    size_t n = seg_count((size_t)r->N);
    if (r->sigma)
        n += seg_count(ke);
    if (r->type == SSA_REQ_DECOMPOSE_RECON && r->groups)
        n += seg_count(2 * (size_t)r->N);
    if (r->type == SSA_REQ_DECOMPOSE_WCORR && r->W)
        n += seg_count(ke * ke);
    return n;
}

static void seg_add(ssa_copy_seg *t, size_t *ns, const double *src, double *dst, size_t n)
{
    while (n > 0)
    {
        const size_t m = n < SRV_SEG_CHUNK ? n : SRV_SEG_CHUNK;
        t[*ns].src = src;
        t[*ns].dst = dst;
        t[*ns].n = (long long)m;
        (*ns)++;
        src += m;
        dst += m;
        n -= m;
    }
}

/* ---- resident store ------------------------------------------------------------------------ */

static res_entry *res_find(ssa_server *s, int id)
{
    res_entry *e = s->htab[(unsigned)id % (unsigned)s->hcap];
    while (e && e->id != id)
        e = e->hnext;
    return e;
}

static void lru_unlink(ssa_server *s, res_entry *e)
{
    if (e->prev)
        e->prev->next = e->next;
    else
        s->lru_head = e->next;
    if (e->next)
        e->next->prev = e->prev;
    else
        s->lru_tail = e->prev;
    e->prev = e->next = NULL;
}

static void lru_front(ssa_server *s, res_entry *e)
{
    e->next = s->lru_head;
    e->prev = NULL;
    if (s->lru_head)
        s->lru_head->prev = e;
    s->lru_head = e;
    if (!s->lru_tail)
        s->lru_tail = e;
}

#define RA_ALIGN ((size_t)256)
#define RA_NONE ((size_t)-1)

/* First fit over the free spans (sorted by offset). */
static size_t ra_alloc(ssa_server *s, size_t bytes)
{
    bytes = (bytes + RA_ALIGN - 1) & ~(RA_ALIGN - 1);
    for (int i = 0; i < s->nspans; i++)
        if (s->spans[i].len >= bytes)
        {
            const size_t off = s->spans[i].off;
            s->spans[i].off += bytes;
            s->spans[i].len -= bytes;
            if (s->spans[i].len == 0)
            {
                memmove(&s->spans[i], &s->spans[i + 1], sizeof(s->spans[0]) * (size_t)(s->nspans - i - 1));
                s->nspans--;
            }
            return off;
        }
    return RA_NONE;
}

/* Return a span, merging it with its neighbours. */
static void ra_free(ssa_server *s, size_t off, size_t bytes)
{
    bytes = (bytes + RA_ALIGN - 1) & ~(RA_ALIGN - 1);
    int i = 0;
    while (i < s->nspans && s->spans[i].off < off)
        i++;
    const int merge_prev = i > 0 && s->spans[i - 1].off + s->spans[i - 1].len == off;
    const int merge_next = i < s->nspans && off + bytes == s->spans[i].off;
    if (merge_prev && merge_next)
    {
        s->spans[i - 1].len += bytes + s->spans[i].len;
        memmove(&s->spans[i], &s->spans[i + 1], sizeof(s->spans[0]) * (size_t)(s->nspans - i - 1));
        s->nspans--;
    }
    else if (merge_prev)
        s->spans[i - 1].len += bytes;
    else if (merge_next)
    {
        s->spans[i].off = off;
        s->spans[i].len += bytes;
    }
    else
    {
        if (s->nspans == s->cspans)
        {
            const int c = s->cspans ? 2 * s->cspans : 1024;
            void *a = realloc(s->spans, sizeof(s->spans[0]) * (size_t)c);
            if (!a)
                return; /* the span is lost to the arena: a leak of space, never an overlap */
            s->spans = a;
            s->cspans = c;
        }
        memmove(&s->spans[i + 1], &s->spans[i], sizeof(s->spans[0]) * (size_t)(s->nspans - i));
        s->spans[i].off = off;
        s->spans[i].len = bytes;
        s->nspans++;
    }
}

static void res_remove(ssa_server *s, res_entry *e)
{
    res_entry **pp = &s->htab[(unsigned)e->id % (unsigned)s->hcap];
    while (*pp && *pp != e)
        pp = &(*pp)->hnext;
    if (*pp)
        *pp = e->hnext;
    lru_unlink(s, e);
    if (e->d && e->aoff != RA_NONE)
        ra_free(s, e->aoff, e->bytes);
    else if (e->d)
        cudaFreeAsync(e->d, s->pool_st);
    s->res_bytes -= e->bytes;
    free(e);
}

/* Evict least recently used entries that nothing uses until `need` more bytes fit. */
static int res_make_room(ssa_server *s, size_t need)
{
    res_entry *e = s->lru_tail;
    while (s->res_bytes + need > s->res_budget && e)
    {
        res_entry *prev = e->prev;
        if (e->refs == 0 && e->state != RES_PENDING)
        {
            res_remove(s, e);
            s->stats.evictions++;
        }
        e = prev;
    }
    return s->res_bytes + need <= s->res_budget ? 0 : -1;
}

static long long round4ll(long long v) { return (v + 3) & ~3LL; }

/* New pending entry for series `id` of shape (N, L) with k resident components, without device
 * memory yet (replaces an idle older one); follow-ups on the series wait while it is pending. */
static res_entry *res_create(ssa_server *s, int id, int N, int L, int k)
{
    res_entry *old = res_find(s, id);
    if (old)
    {
        if (old->refs > 0 || old->state == RES_PENDING)
            return NULL;
        res_remove(s, old);
    }
    res_entry *e = (res_entry *)calloc(1, sizeof(res_entry));
    if (!e)
        return NULL;
    e->id = id;
    e->L = L;
    e->N = N;
    e->K = N - L + 1;
    e->k = k;
    e->ldL = round4ll(L);
    e->ldK = round4ll(e->K);
    e->state = RES_PENDING;
    unsigned h = (unsigned)id % (unsigned)s->hcap;
    e->hnext = s->htab[h];
    s->htab[h] = e;
    lru_front(s, e);
    return e;
}

/* Doubles before the factor floats of an entry's block (a multiple of 2, so the floats start
 * 16-byte aligned). */
static size_t res_dbl(const res_entry *e)
{
    const size_t n = 2 * (size_t)(e->L - 1) + 1 + (size_t)e->k + (size_t)e->N;
    return (n + 1) & ~(size_t)1;
}

/* Device memory for a pending entry when its decomposition is launched (layout in res_entry),
 * evicting least recently used idle series beyond the resident budget. */
static int res_alloc(ssa_server *s, res_entry *e)
{
    const size_t nd = res_dbl(e);
    const size_t bytes = sizeof(double) * nd + sizeof(float) * (size_t)(e->ldL + e->ldK) * (size_t)e->k;
    if (res_make_room(s, bytes) != 0)
        return -1;
    e->aoff = RA_NONE;
    if (s->res_arena)
    {
        /* evict further least recently used idle series while fragmentation leaves no span */
        size_t off;
        while ((off = ra_alloc(s, bytes)) == RA_NONE)
        {
            res_entry *v = s->lru_tail;
            while (v && (v->refs > 0 || v->state == RES_PENDING || v == e))
                v = v->prev;
            if (!v)
                return -1;
            res_remove(s, v);
            s->stats.evictions++;
        }
        e->aoff = off;
        e->d = (double *)(s->res_arena + off);
    }
    else
    {
        cudaMemPool_t pool = ssar_pool();
        if (!pool || cudaMallocFromPoolAsync((void **)&e->d, bytes, pool, s->pool_st) != cudaSuccess)
        {
            e->d = NULL;
            return -1;
        }
    }
    e->sig = e->d + 2 * (size_t)(e->L - 1) + 1;
    e->x = e->sig + e->k;
    e->U = (float *)(e->d + nd);
    e->V = e->U + e->ldL * e->k;
    e->bytes = bytes;
    s->res_bytes += bytes;
    return 0;
}

/* ---- helpers ------------------------------------------------------------------------------ */

/* SSA_SERVER_TRACE=1 in the environment: batch launches that take the worker over 5 ms are
 * reported on stderr with their phases (a diagnostic for latency tails). */
static int srv_trace(void)
{
    static int v = -1;
    if (v < 0)
    {
        const char *e = getenv("SSA_SERVER_TRACE");
        v = e && e[0] == '1';
    }
    return v;
}

static int grow_host(void **p, size_t *cap, size_t need, size_t elem)
{
    if (need <= *cap && *p)
        return 0;
    if (*p)
        cudaFreeHost(*p);
    *p = NULL;
    *cap = 0;
    size_t n = need + need / 4 + 16;
    if (cudaMallocHost(p, n * elem) != cudaSuccess)
        return -1;
    *cap = n;
    return 0;
}

static int grow_dev(void **p, size_t *cap, size_t need, size_t elem)
{
    if (need <= *cap && *p)
        return 0;
    if (*p)
        cudaFree(*p);
    *p = NULL;
    *cap = 0;
    size_t n = need + need / 4 + 16;
    if (cudaMalloc(p, n * elem) != cudaSuccess)
        return -1;
    *cap = n;
    return 0;
}

static int ensure_cap(void ***arr, int *cap, int need, size_t elem)
{
    if (need <= *cap)
        return 0;
    int n = need + need / 2 + 8;
    void **a = (void **)realloc(*arr, elem * (size_t)n);
    if (!a)
        return -1;
    *arr = a;
    *cap = n;
    return 0;
}

static void finish_request(ssa_server *s, ssa_request *r, int status)
{
    r->status = status;
    r->t_done = ssa_server_now();
    pthread_mutex_lock(&s->mu);
    s->outstanding--;
    if (status == 0)
        s->stats.completed++;
    else
        s->stats.failed++;
    pthread_cond_broadcast(&s->cv_done);
    pthread_mutex_unlock(&s->mu);
}

static int is_decomp(const ssa_request *r) { return r->type == SSA_REQ_DECOMPOSE_RECON || r->type == SSA_REQ_DECOMPOSE_WCORR; }

static int valid_decomp(const ssa_server *s, const ssa_request *r)
{
    if (!r->x || r->N < 4 || r->L < 2 || r->L > r->N - 1 || r->k < 1 || ssad_logh_for(r->N) > SSA_MAX_LOGH_ALL)
        return 0;
    const int K = r->N - r->L + 1;
    return imin(r->k + s->p, imin(r->L, K)) <= SSA_MAX_KP;
}

/* ---- decomposition batches ------------------------------------------------------------------ */

static int slot_reserve(slot_t *sl, int n)
{
    if (n <= sl->cap)
        return 0;
    int c = n + n / 2 + 16;
    void *a[8];
    a[0] = realloc(sl->req, sizeof(ssa_request *) * c);
    if (a[0])
        sl->req = (ssa_request **)a[0];
    a[1] = realloc(sl->N, sizeof(int) * c);
    if (a[1])
        sl->N = (int *)a[1];
    a[2] = realloc(sl->L, sizeof(int) * c);
    if (a[2])
        sl->L = (int *)a[2];
    a[3] = realloc(sl->k, sizeof(int) * c);
    if (a[3])
        sl->k = (int *)a[3];
    a[4] = realloc(sl->seeds, sizeof(unsigned long long) * c);
    if (a[4])
        sl->seeds = (unsigned long long *)a[4];
    a[5] = realloc(sl->lrf_dst, sizeof(double *) * c);
    if (a[5])
        sl->lrf_dst = (double **)a[5];
    a[6] = realloc(sl->res, sizeof(res_entry *) * c);
    if (a[6])
        sl->res = (res_entry **)a[6];
    a[7] = realloc(sl->wantw, sizeof(unsigned char) * c);
    if (a[7])
        sl->wantw = (unsigned char *)a[7];
    for (int i = 0; i < 8; i++)
        if (!a[i])
            return -1;
    size_t *z[3] = {NULL, NULL, NULL};
    z[0] = (size_t *)realloc(sl->xoff, sizeof(size_t) * c);
    if (z[0])
        sl->xoff = z[0];
    z[1] = (size_t *)realloc(sl->sin, sizeof(size_t) * c);
    if (z[1])
        sl->sin = z[1];
    z[2] = (size_t *)realloc(sl->sout, sizeof(size_t) * c);
    if (z[2])
        sl->sout = z[2];
    if (!z[0] || !z[1] || !z[2])
        return -1;
    double **h = (double **)realloc(sl->hp, sizeof(double *) * 4 * (size_t)c);
    if (!h)
        return -1;
    sl->hp = h;
    sl->cap = c;
    return 0;
}

/* Order the gathered batch by FFT-length bucket (arrival order kept within a bucket) and record
 * the bucket ranges. Every request carries its own seed and buffers, so the order changes no
 * result. */
static int slot_order(slot_t *sl)
{
    const int n = sl->n;
    int cnt[SSAR_NB + 1] = {0};
    int *bk = (int *)malloc(sizeof(int) * (size_t)n), *pos = (int *)malloc(sizeof(int) * (size_t)n);
    void *tmp = malloc((sizeof(void *) * 4 + sizeof(size_t)) * (size_t)n);
    if (!bk || !pos || !tmp)
    {
        free(bk);
        free(pos);
        free(tmp);
        return -1;
    }
    for (int i = 0; i < n; i++)
    {
        bk[i] = ssar_bucket_index(sl->N[i]);
        cnt[bk[i] + 1]++;
    }
    for (int g = 0; g < SSAR_NB; g++)
        cnt[g + 1] += cnt[g];
    sl->nrange = 0;
    for (int g = 0; g < SSAR_NB; g++)
        if (cnt[g + 1] > cnt[g])
        {
            sl->rlo[sl->nrange] = cnt[g];
            sl->rhi[sl->nrange] = cnt[g + 1];
            sl->rdone[sl->nrange] = 0;
            sl->nrange++;
        }
    for (int i = 0; i < n; i++)
        pos[i] = cnt[bk[i]]++;
#define SRV_PERMUTE(arr, T)                                 \
    do                                                      \
    {                                                       \
        T *t_ = (T *)tmp;                                   \
        for (int i_ = 0; i_ < n; i_++)                      \
            t_[pos[i_]] = (arr)[i_];                        \
        memcpy((arr), t_, sizeof(T) * (size_t)n);           \
    } while (0)
    SRV_PERMUTE(sl->req, ssa_request *);
    SRV_PERMUTE(sl->N, int);
    SRV_PERMUTE(sl->L, int);
    SRV_PERMUTE(sl->k, int);
    SRV_PERMUTE(sl->seeds, unsigned long long);
    SRV_PERMUTE(sl->lrf_dst, double *);
    SRV_PERMUTE(sl->res, res_entry *);
    SRV_PERMUTE(sl->wantw, unsigned char);
    SRV_PERMUTE(sl->sin, size_t);
    SRV_PERMUTE(sl->sout, size_t);
#undef SRV_PERMUTE
    {
        double **t4 = (double **)tmp;
        for (int i = 0; i < n; i++)
            memcpy(t4 + 4 * (size_t)pos[i], sl->hp + 4 * (size_t)i, sizeof(double *) * 4);
        memcpy(sl->hp, t4, sizeof(double *) * 4 * (size_t)n);
    }
    free(bk);
    free(pos);
    free(tmp);
    return 0;
}

/* Launch the batch gathered in sl (sl->n requests, dims and staging offsets filled). */
static int slot_launch(ssa_server *s, slot_t *sl)
{
    const double t0 = ssa_server_now();
    sl->nrange = 0;
    if (slot_order(sl) != 0)
        return -1;
    size_t nx = 0;
    for (int i = 0; i < sl->n; i++)
    {
        sl->xoff[i] = nx;
        nx += (size_t)sl->N[i];
    }
    cudaStream_t ms = ssar_main_stream(sl->rb);
    if (sl->c_dx < nx)
    {
        /* stream-ordered, so that growing does not wait for the other slots' work */
        if (sl->d_x)
            cudaFreeAsync(sl->d_x, ms);
        sl->d_x = NULL;
        sl->c_dx = 0;
        if (cudaMallocFromPoolAsync((void **)&sl->d_x, sizeof(double) * (nx + nx / 4), ssar_pool(), ms) != cudaSuccess)
            return -1;
        sl->c_dx = nx + nx / 4;
    }
    /* resident blocks were allocated on the pool stream: order the batch after them */
    if (cudaEventRecord(s->ev_pool, s->pool_st) != cudaSuccess || cudaStreamWaitEvent(ms, s->ev_pool, 0) != cudaSuccess)
        return -1;
    /* the copy kernel's segment table; the slot is idle, so its table is free */
    size_t nseg = 0;
    for (int i = 0; i < sl->n; i++)
    {
        nseg += req_segs(s, sl->req[i]);
        const res_entry *e = sl->res[i];
        if (e && e->d)
            nseg += seg_count((size_t)e->k) + seg_count((size_t)e->N) + seg_count((size_t)(e->ldL * e->k / 2)) +
                    seg_count((size_t)(e->ldK * e->k / 2));
    }
    if (nseg > sl->c_seg)
    {
        if (sl->h_seg)
            cudaFreeHost(sl->h_seg);
        sl->h_seg = sl->h_seg_d = NULL;
        sl->c_seg = 0;
        if (cudaMallocHost((void **)&sl->h_seg, sizeof(ssa_copy_seg) * (2 * nseg + 1024)) != cudaSuccess ||
            !(sl->h_seg_d = (ssa_copy_seg *)mapped(sl->h_seg)))
            return -1;
        sl->c_seg = 2 * nseg + 1024;
    }
    /* inputs: one gather launch reading the callers' page-locked buffers, and the staging area
     * that the pageable ones are copied into */
    size_t ns = 0;
    for (int i = 0; i < sl->n; i++)
    {
        const ssa_request *r = sl->req[i];
        const double *src = sl->hp[4 * i];
        if (!src)
        {
            memcpy(sl->h_in + sl->sin[i], r->x, sizeof(double) * r->N);
            src = sl->h_in_d + sl->sin[i];
        }
        seg_add(sl->h_seg, &ns, src, sl->d_x + sl->xoff[i], (size_t)r->N);
    }
    const size_t nin = ns;
    if (ssad_copy_segments(sl->h_seg_d, (int)nin, ms) != 0)
        return -1;
    const double t1 = ssa_server_now();
    if (ssar_run_enqueue_ex(sl->rb, sl->n, sl->N, sl->L, sl->k, sl->d_x, sl->seeds, sl->lrf_dst, sl->wantw) != 0)
        return -1;
    const double t2 = ssa_server_now();
    /* outputs the requests ask for, per FFT-length bucket on its stream: one scatter launch writing
     * the callers' page-locked buffers, or the staging area finish_range copies from */
    const size_t *off = ssar_offsets(sl->rb);
    const double *dsig = ssar_sigma(sl->rb), *dW = ssar_W(sl->rb), *dg = ssar_groups(sl->rb);
    const int *dst = ssar_status(sl->rb), *dlst = ssar_lrf_status(sl->rb);
    for (int rg = 0; rg < sl->nrange; rg++)
    {
        const int lo = sl->rlo[rg], hi = sl->rhi[rg];
        cudaStream_t bs = ssar_bucket_stream(sl->rb, ssar_bucket_index(sl->N[lo]));
        if (!bs)
            return -1;
        const size_t seg0 = ns;
        for (int i = lo; i < hi; i++)
        {
            ssa_request *r = sl->req[i];
            const size_t ke = (size_t)req_kout(s, r);
            const int direct = sl->sout[i] == SRV_DIRECT;
            size_t so = sl->sout[i];
            if (r->sigma)
            {
                seg_add(sl->h_seg, &ns, dsig + off[4 * i + 1], direct ? sl->hp[4 * i + 1] : sl->h_out_d + so, ke);
                so += ke;
            }
            if (r->type == SSA_REQ_DECOMPOSE_RECON && r->groups)
                seg_add(sl->h_seg, &ns, dg + off[4 * i + 3], direct ? sl->hp[4 * i + 2] : sl->h_out_d + so,
                        2 * (size_t)r->N);
            if (r->type == SSA_REQ_DECOMPOSE_WCORR && r->W)
                seg_add(sl->h_seg, &ns, dW + off[4 * i + 2], direct ? sl->hp[4 * i + 3] : sl->h_out_d + so, ke * ke);
            /* the series stays resident: sigma, signal and the factor blocks (floats copied as pairs;
             * both leading dimensions are multiples of 4) */
            res_entry *e = sl->res[i];
            const float *U = NULL, *V = NULL;
            if (e && e->d && ssar_series_factors(sl->rb, i, &U, &V) == e->k)
            {
                seg_add(sl->h_seg, &ns, dsig + off[4 * i + 1], e->sig, (size_t)e->k);
                seg_add(sl->h_seg, &ns, sl->d_x + sl->xoff[i], e->x, (size_t)e->N);
                seg_add(sl->h_seg, &ns, (const double *)U, (double *)e->U, (size_t)(e->ldL * e->k / 2));
                seg_add(sl->h_seg, &ns, (const double *)V, (double *)e->V, (size_t)(e->ldK * e->k / 2));
            }
        }
        /* the bucket's outputs and status words, on its stream right after its part of the run */
        if (ssad_copy_segments(sl->h_seg_d + seg0, (int)(ns - seg0), bs) != 0 ||
            cudaMemcpyAsync(sl->h_st + lo, dst + lo, sizeof(int) * (size_t)(hi - lo), cudaMemcpyDeviceToHost, bs) !=
                cudaSuccess ||
            cudaMemcpyAsync(sl->h_lst + lo, dlst + lo, sizeof(int) * (size_t)(hi - lo), cudaMemcpyDeviceToHost, bs) !=
                cudaSuccess ||
            cudaEventRecord(sl->rev[rg], bs) != cudaSuccess || cudaStreamWaitEvent(ms, sl->rev[rg], 0) != cudaSuccess)
            return -1;
    }
    if (cudaEventRecord(sl->done, ms) != cudaSuccess)
        return -1;
    sl->busy = 1;
    s->stats.batches++;
    s->stats.decompositions += sl->n;
    if (sl->n > s->stats.max_batch)
        s->stats.max_batch = sl->n;
    const double dt = ssa_server_now() - t0;
    s->stats.host_launch_s += dt;
    if (dt > s->stats.host_launch_max_s)
        s->stats.host_launch_max_s = dt;
    if (srv_trace() && dt > 5e-3)
        fprintf(stderr, "ssa_server: batch of %d formed in %.1f ms (inputs %.1f, enqueue %.1f, outputs %.1f)\n", sl->n,
                1e3 * dt, 1e3 * (t1 - t0), 1e3 * (t2 - t1), 1e3 * (dt - (t2 - t0)));
    return 0;
}

/* Complete requests lo .. hi - 1 of the slot's batch (their outputs and status words are on
 * the host). */
static void finish_range(ssa_server *s, slot_t *sl, int lo, int hi, int launch_ok)
{
    const double t0 = ssa_server_now();
    for (int i = lo; i < hi; i++)
    {
        ssa_request *r = sl->req[i];
        int ok = launch_ok && sl->h_st[i] == 0;
        if (ok)
        {
            const int ke = req_kout(s, r);
            r->k_out = ke;
            if (sl->sout[i] != SRV_DIRECT)
            {
                size_t so = sl->sout[i];
                if (r->sigma)
                {
                    memcpy(r->sigma, sl->h_out + so, sizeof(double) * ke);
                    so += (size_t)ke;
                }
                if (r->type == SSA_REQ_DECOMPOSE_RECON && r->groups)
                    memcpy(r->groups, sl->h_out + so, sizeof(double) * 2 * r->N);
                if (r->type == SSA_REQ_DECOMPOSE_WCORR && r->W)
                    memcpy(r->W, sl->h_out + so, sizeof(double) * ke * ke);
            }
        }
        res_entry *e = sl->res[i];
        if (e)
        {
            e->state = (ok && e->d && r->k_out == e->k) ? RES_READY : RES_FAILED;
            /* the default forecast group [0, 1, 2] needs at least 3 components */
            e->lrf_ok = sl->h_lst[i] == 0 && r->k_out > 2;
        }
        finish_request(s, r, ok ? 0 : -1);
    }
    s->stats.host_finish_s += ssa_server_now() - t0;
}

static void slot_release(slot_t *sl)
{
    sl->n = 0;
    sl->nrange = 0;
    sl->busy = 0;
    sl->in_used = sl->out_used = 0;
}

/* Complete every request of the batch not completed yet and free the slot. */
static void slot_finish(ssa_server *s, slot_t *sl, int launch_ok)
{
    if (sl->nrange == 0)
        finish_range(s, sl, 0, sl->n, launch_ok);
    for (int r = 0; r < sl->nrange; r++)
        if (!sl->rdone[r])
        {
            finish_range(s, sl, sl->rlo[r], sl->rhi[r], launch_ok);
            sl->rdone[r] = 1;
        }
    slot_release(sl);
}

/* ---- forecast batches ------------------------------------------------------------------- */

static int fs_launch(ssa_server *s)
{
    fslot_t *f = &s->fs;
    size_t nout = 0;
    for (int i = 0; i < f->n; i++)
        nout += (size_t)f->req[i]->h;
    if (grow_dev((void **)&f->d_out, &f->c_dout, nout, sizeof(double)) != 0)
        return -1;
    if (grow_host((void **)&f->h_out, &f->c_hout, nout, sizeof(double)) != 0)
        return -1;
    size_t o = 0;
    for (int i = 0; i < f->n; i++)
    {
        ssa_fc_job *J = &f->h_jobs[i];
        res_entry *e = f->res[i];
        J->R = e->d;
        J->tail = e->d + (e->L - 1);
        J->out = f->d_out + o;
        J->w = e->L - 1;
        J->h = f->req[i]->h;
        o += (size_t)J->h;
    }
    if (cudaMemcpyAsync(f->d_jobs, f->h_jobs, sizeof(ssa_fc_job) * f->n, cudaMemcpyHostToDevice, f->st) !=
            cudaSuccess ||
        ssad_forecast_apply(f->d_jobs, f->n, f->st) != 0 ||
        cudaMemcpyAsync(f->h_out, f->d_out, sizeof(double) * nout, cudaMemcpyDeviceToHost, f->st) != cudaSuccess ||
        cudaEventRecord(f->done, f->st) != cudaSuccess)
        return -1;
    f->busy = 1;
    s->stats.forecast_batches++;
    s->stats.forecasts += f->n;
    return 0;
}

static void fs_finish(ssa_server *s, int ok)
{
    fslot_t *f = &s->fs;
    size_t o = 0;
    for (int i = 0; i < f->n; i++)
    {
        ssa_request *r = f->req[i];
        if (ok && r->forecast)
            memcpy(r->forecast, f->h_out + o, sizeof(double) * r->h);
        o += (size_t)r->h;
        f->res[i]->refs--;
        finish_request(s, r, ok ? 0 : -1);
    }
    f->n = 0;
    f->busy = 0;
}

/* ---- follow-up batches on resident factors ---------------------------------------------------- */

static int is_followup(const ssa_request *r)
{
    return r->type == SSA_REQ_RECONSTRUCT || (r->type == SSA_REQ_FORECAST && r->group) ||
           (r->type == SSA_REQ_CADZOW && !r->x);
}

static int us_reserve(uslot_t *u, int n)
{
    if (n <= u->cap)
        return 0;
    const int c = n + n / 2 + 16;
    void *p[13];
    p[0] = realloc(u->req, sizeof(ssa_request *) * c);
    if (p[0])
        u->req = (ssa_request **)p[0];
    p[1] = realloc(u->res, sizeof(res_entry *) * c);
    if (p[1])
        u->res = (res_entry **)p[1];
    p[2] = realloc(u->N, sizeof(int) * c);
    if (p[2])
        u->N = (int *)p[2];
    p[3] = realloc(u->L, sizeof(int) * c);
    if (p[3])
        u->L = (int *)p[3];
    p[4] = realloc(u->k, sizeof(int) * c);
    if (p[4])
        u->k = (int *)p[4];
    p[5] = realloc(u->goff, sizeof(int) * (c + 1));
    if (p[5])
        u->goff = (int *)p[5];
    p[6] = realloc((void *)u->U, sizeof(float *) * c);
    if (p[6])
        u->U = (const float **)p[6];
    p[7] = realloc((void *)u->V, sizeof(float *) * c);
    if (p[7])
        u->V = (const float **)p[7];
    p[8] = realloc((void *)u->sig, sizeof(double *) * c);
    if (p[8])
        u->sig = (const double **)p[8];
    p[9] = realloc(u->lrf, sizeof(double *) * c);
    if (p[9])
        u->lrf = (double **)p[9];
    p[10] = realloc(u->tmpoff, sizeof(size_t) * c);
    if (p[10])
        u->tmpoff = (size_t *)p[10];
    p[11] = realloc(u->hoff, sizeof(size_t) * c);
    if (p[11])
        u->hoff = (size_t *)p[11];
    p[12] = NULL;
    for (int i = 0; i < 12; i++)
        if (!p[i])
            return -1;
    int *h = NULL;
    if (cudaMallocHost((void **)&h, sizeof(int) * c) != cudaSuccess)
        return -1;
    if (u->h_lst)
        cudaFreeHost(u->h_lst);
    u->h_lst = h;
    u->cap = c;
    return 0;
}

/* Host doubles of a follow-up's outputs in the pinned area: the group reconstruction (N) for
 * reconstructions and Cadzow (plus the resident signal, N, for Cadzow), h forecasts. */
static size_t us_out_doubles(const ssa_request *r, const res_entry *e)
{
    if (r->type == SSA_REQ_FORECAST)
        return (size_t)r->h;
    return (size_t)e->N * (r->type == SSA_REQ_CADZOW ? 2 : 1);
}

static int us_launch(ssa_server *s)
{
    uslot_t *u = &s->us;
    cudaStream_t st = ssar_main_stream(u->rb);
    int ng = 0, nfc = 0;
    size_t ntmp = 0, nfcout = 0, nout = 0;
    for (int i = 0; i < u->n; i++)
    {
        const ssa_request *r = u->req[i];
        ng += r->type == SSA_REQ_CADZOW ? r->rank : r->n_group;
        if (r->type == SSA_REQ_FORECAST)
        {
            nfc++;
            ntmp += 2 * (size_t)(u->res[i]->L - 1) + 1;
            nfcout += (size_t)r->h;
        }
        nout += us_out_doubles(r, u->res[i]);
    }
    if (ng > u->cgidx)
    {
        int *g = (int *)realloc(u->gidx, sizeof(int) * (size_t)(ng + ng / 2 + 16));
        if (!g)
            return -1;
        u->gidx = g;
        u->cgidx = ng + ng / 2 + 16;
    }
    if (grow_dev((void **)&u->d_tmp, &u->c_tmp, ntmp + 1, sizeof(double)) != 0 ||
        grow_dev((void **)&u->d_fcout, &u->c_fcout, nfcout + 1, sizeof(double)) != 0 ||
        grow_host((void **)&u->h_out, &u->c_hout, nout + 1, sizeof(double)) != 0)
        return -1;
    if (nfc > u->c_fc)
    {
        ssa_fc_job *hj = NULL, *dj = NULL;
        const int c = nfc + nfc / 2 + 16;
        if (cudaMallocHost((void **)&hj, sizeof(ssa_fc_job) * c) != cudaSuccess ||
            cudaMalloc((void **)&dj, sizeof(ssa_fc_job) * c) != cudaSuccess)
        {
            if (hj)
                cudaFreeHost(hj);
            return -1;
        }
        if (u->h_fc)
            cudaFreeHost(u->h_fc);
        if (u->d_fc)
            cudaFree(u->d_fc);
        u->h_fc = hj;
        u->d_fc = dj;
        u->c_fc = c;
    }
    size_t otmp = 0, ofc = 0, oh = 0;
    int og = 0, jf = 0;
    for (int i = 0; i < u->n; i++)
    {
        const ssa_request *r = u->req[i];
        const res_entry *e = u->res[i];
        u->N[i] = e->N;
        u->L[i] = e->L;
        u->k[i] = e->k;
        u->U[i] = e->U;
        u->V[i] = e->V;
        u->sig[i] = e->sig;
        u->goff[i] = og;
        if (r->type == SSA_REQ_CADZOW)
            for (int j = 0; j < r->rank; j++)
                u->gidx[og++] = j;
        else
            for (int j = 0; j < r->n_group; j++)
                u->gidx[og++] = r->group[j];
        u->lrf[i] = NULL;
        u->hoff[i] = oh;
        oh += us_out_doubles(r, e);
        if (r->type == SSA_REQ_FORECAST)
        {
            u->tmpoff[i] = otmp;
            u->lrf[i] = u->d_tmp + otmp;
            ssa_fc_job *J = &u->h_fc[jf++];
            J->R = u->d_tmp + otmp;
            J->tail = u->d_tmp + otmp + (e->L - 1);
            J->out = u->d_fcout + ofc;
            J->w = e->L - 1;
            J->h = r->h;
            otmp += 2 * (size_t)(e->L - 1) + 1;
            ofc += (size_t)r->h;
        }
    }
    u->goff[u->n] = og;
    /* the resident blocks were allocated on the pool stream */
    if (cudaEventRecord(s->ev_pool, s->pool_st) != cudaSuccess || cudaStreamWaitEvent(st, s->ev_pool, 0) != cudaSuccess)
        return -1;
    if (ssar_run_followup(u->rb, u->n, u->N, u->L, u->k, (const float *const *)u->U, (const float *const *)u->V,
                          (const double *const *)u->sig, u->gidx, u->goff, u->lrf) != 0)
        return -1;
    if (nfc > 0 && (cudaMemcpyAsync(u->d_fc, u->h_fc, sizeof(ssa_fc_job) * nfc, cudaMemcpyHostToDevice, st) !=
                        cudaSuccess ||
                    ssad_forecast_apply(u->d_fc, nfc, st) != 0))
        return -1;
    const size_t *off = ssar_offsets(u->rb);
    const double *dg = ssar_groups(u->rb);
    ofc = 0;
    for (int i = 0; i < u->n; i++)
    {
        const ssa_request *r = u->req[i];
        const res_entry *e = u->res[i];
        double *h = u->h_out + u->hoff[i];
        cudaError_t c = cudaSuccess;
        if (r->type == SSA_REQ_FORECAST)
        {
            c = cudaMemcpyAsync(h, u->d_fcout + ofc, sizeof(double) * r->h, cudaMemcpyDeviceToHost, st);
            ofc += (size_t)r->h;
        }
        else
        {
            c = cudaMemcpyAsync(h, dg + off[4 * i + 3], sizeof(double) * e->N, cudaMemcpyDeviceToHost, st);
            if (c == cudaSuccess && r->type == SSA_REQ_CADZOW)
                c = cudaMemcpyAsync(h + e->N, e->x, sizeof(double) * e->N, cudaMemcpyDeviceToHost, st);
        }
        if (c != cudaSuccess)
            return -1;
    }
    if (cudaMemcpyAsync(u->h_lst, ssar_lrf_status(u->rb), sizeof(int) * u->n, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaEventRecord(u->done, st) != cudaSuccess)
        return -1;
    u->busy = 1;
    s->stats.followup_batches++;
    s->stats.followups += u->n;
    return 0;
}

static void cz_push(ssa_server *s, ssa_request *r, double *x, double *y1);

static void us_finish(ssa_server *s, int ok)
{
    uslot_t *u = &s->us;
    for (int i = 0; i < u->n; i++)
    {
        ssa_request *r = u->req[i];
        res_entry *e = u->res[i];
        const double *h = u->h_out + u->hoff[i];
        int st = ok ? 0 : -1;
        if (ok && r->type == SSA_REQ_RECONSTRUCT)
        {
            if (r->out)
                memcpy(r->out, h, sizeof(double) * e->N);
        }
        else if (ok && r->type == SSA_REQ_FORECAST)
        {
            if (u->h_lst[i] != 0)
                st = -1; /* verticality >= 1: no LRF */
            else if (r->forecast)
                memcpy(r->forecast, h, sizeof(double) * r->h);
        }
        else if (ok && r->type == SSA_REQ_CADZOW)
        {
            double *x = (double *)malloc(sizeof(double) * e->N), *y1 = (double *)malloc(sizeof(double) * e->N);
            if (x && y1)
            {
                memcpy(y1, h, sizeof(double) * e->N);
                memcpy(x, h + e->N, sizeof(double) * e->N);
                r->N = e->N;
                r->L = e->L;
                e->refs--;
                cz_push(s, r, x, y1); /* finished by the Cadzow worker */
                continue;
            }
            free(x);
            free(y1);
            st = -1;
        }
        e->refs--;
        finish_request(s, r, st);
    }
    u->n = 0;
    u->busy = 0;
}

/* ---- Cadzow worker ------------------------------------------------------------------------------ */

static void cz_push(ssa_server *s, ssa_request *r, double *x, double *y1)
{
    cz_item *it = (cz_item *)calloc(1, sizeof(cz_item));
    if (!it)
    {
        free(x);
        free(y1);
        finish_request(s, r, -1);
        return;
    }
    it->r = r;
    it->x = x;
    it->y1 = y1;
    pthread_mutex_lock(&s->mu);
    if (s->cz_tail)
        s->cz_tail->next = it;
    else
        s->cz_head = it;
    s->cz_tail = it;
    pthread_cond_signal(&s->cz_cv);
    pthread_mutex_unlock(&s->mu);
}

/* Runs Cadzow requests one after another: a request with its own signal from the start, one on a
 * resident series from the projection its follow-up batch made out of the resident factors. */
static void *cz_worker(void *arg)
{
    ssa_server *s = (ssa_server *)arg;
    cudaSetDevice(s->device);
    for (;;)
    {
        pthread_mutex_lock(&s->mu);
        while (!s->cz_head && !s->cz_stop)
            pthread_cond_wait(&s->cz_cv, &s->mu);
        cz_item *it = s->cz_head;
        if (!it)
        {
            pthread_mutex_unlock(&s->mu);
            break;
        }
        s->cz_head = it->next;
        if (!s->cz_head)
            s->cz_tail = NULL;
        pthread_mutex_unlock(&s->mu);
        ssa_request *r = it->r;
        SSA_CadzowResult res;
        memset(&res, 0, sizeof(res));
        const double *x = it->x ? it->x : r->x;
        double *out = r->out ? r->out : (double *)malloc(sizeof(double) * (size_t)r->N);
        const int rc = out ? ssab_cadzow_from(x, it->y1, r->N, r->L, r->rank, r->max_iter, r->tol, out, &res) : -1;
        if (!r->out)
            free(out);
        r->iterations = res.iterations;
        r->final_diff = res.final_diff;
        pthread_mutex_lock(&s->mu);
        s->stats.cadzow_requests++;
        if (rc >= 0)
            s->stats.cadzow_iterations += res.iterations;
        pthread_mutex_unlock(&s->mu);
        free(it->x);
        free(it->y1);
        free(it);
        finish_request(s, r, rc >= 0 ? 0 : -1);
    }
    return NULL;
}

/* ---- worker ---------------------------------------------------------------------------------- */

static int poll_done(ssa_server *s)
{
    int progressed = 0;
    for (int i = 0; i < s->nslots; i++)
    {
        slot_t *sl = &s->slots[i];
        if (!sl->busy)
            continue;
        /* buckets that are done complete their requests now */
        int open = 0;
        for (int r = 0; r < sl->nrange; r++)
        {
            if (sl->rdone[r])
                continue;
            const cudaError_t qr = cudaEventQuery(sl->rev[r]);
            if (qr == cudaErrorNotReady)
            {
                open++;
                continue;
            }
            finish_range(s, sl, sl->rlo[r], sl->rhi[r], qr == cudaSuccess);
            sl->rdone[r] = 1;
            progressed = 1;
        }
        if (open)
            continue;
        cudaError_t q = cudaEventQuery(sl->done);
        if (q == cudaErrorNotReady)
            continue;
        slot_finish(s, sl, q == cudaSuccess);
        progressed = 1;
    }
    if (s->fs.busy)
    {
        cudaError_t q = cudaEventQuery(s->fs.done);
        if (q != cudaErrorNotReady)
        {
            fs_finish(s, q == cudaSuccess);
            progressed = 1;
        }
    }
    if (s->us.busy)
    {
        cudaError_t q = cudaEventQuery(s->us.done);
        if (q != cudaErrorNotReady)
        {
            us_finish(s, q == cudaSuccess);
            progressed = 1;
        }
    }
    return progressed;
}

/* Move submitted requests to the worker's pending list (arrival order kept). */
static void take_queue(ssa_server *s)
{
    pthread_mutex_lock(&s->mu);
    if (s->qcount > 0 && ensure_cap((void ***)&s->pend, &s->cpend, s->npend + s->qcount, sizeof(ssa_request *)) == 0)
    {
        while (s->qcount > 0)
        {
            s->pend[s->npend++] = s->q[s->qhead];
            s->qhead = (s->qhead + 1) % s->qcap;
            s->qcount--;
        }
    }
    pthread_mutex_unlock(&s->mu);
}

/* Size class of a decomposition: series whose transforms run on thread-block clusters (real FFT
 * length above 32768) take several times longer than the rest, and a batch slot is busy until
 * its last bucket is done, so they are batched apart: a short series never waits for a long
 * one's slot. Within a class requests keep their arrival order. */
#define SRV_LONG_N 32768
static int srv_class(const ssa_request *r) { return r->N > SRV_LONG_N; }

/* Form and launch at most one forecast batch and one decomposition batch per free slot. */
static int dispatch(ssa_server *s)
{
    int progressed = 0;
    slot_t *free_slot = NULL;
    for (int i = 0; i < s->nslots && !free_slot; i++)
        if (!s->slots[i].busy)
            free_slot = &s->slots[i];
    fslot_t *f = s->fs.busy ? NULL : &s->fs;
    uslot_t *u = s->us.busy ? NULL : &s->us;
    size_t bytes = 0;
    int kept = 0;
    int cls = -1; /* size class of the batch being formed */
    for (int i = 0; i < s->npend; i++)
    {
        ssa_request *r = s->pend[i];
        int keep = 1;
        if (r->type == SSA_REQ_FORECAST && !r->group)
        {
            res_entry *e = res_find(s, r->series_id);
            if (!e || e->state == RES_FAILED || (e->state == RES_READY && !e->lrf_ok) || r->h < 1 ||
                r->h > SSA_FC_MAX_H)
            {
                finish_request(s, r, -1);
                keep = 0;
                progressed = 1;
            }
            else if (e->state == RES_READY && f && f->n < s->max_batch)
            {
                if (f->n >= f->cap)
                {
                    int c = f->cap ? 2 * f->cap : 256;
                    void *a = realloc(f->req, sizeof(ssa_request *) * c);
                    void *b = a ? realloc(f->res, sizeof(res_entry *) * c) : NULL;
                    if (a)
                        f->req = (ssa_request **)a;
                    if (b)
                        f->res = (res_entry **)b;
                    ssa_fc_job *hj = NULL, *dj = NULL;
                    if (a && b && cudaMallocHost((void **)&hj, sizeof(ssa_fc_job) * c) == cudaSuccess &&
                        cudaMalloc((void **)&dj, sizeof(ssa_fc_job) * c) == cudaSuccess)
                    {
                        if (f->h_jobs)
                            cudaFreeHost(f->h_jobs);
                        if (f->d_jobs)
                            cudaFree(f->d_jobs);
                        f->h_jobs = hj;
                        f->d_jobs = dj;
                        f->cap = c;
                    }
                    else
                    {
                        if (hj)
                            cudaFreeHost(hj);
                        f = NULL; /* try again next round */
                    }
                }
                if (f && f->n < f->cap)
                {
                    e->refs++;
                    lru_unlink(s, e);
                    lru_front(s, e);
                    f->req[f->n] = r;
                    f->res[f->n] = e;
                    f->n++;
                    keep = 0;
                }
            }
        }
        else if (is_followup(r))
        {
            res_entry *e = res_find(s, r->series_id);
            int bad = !e || e->state == RES_FAILED;
            if (!bad && r->type == SSA_REQ_CADZOW)
                bad = r->rank < 1 || r->rank > e->k || r->max_iter < 1;
            else if (!bad)
            {
                int any = 0; /* a group needs at least one component the series has */
                for (int j = 0; r->group && j < r->n_group; j++)
                    any |= r->group[j] >= 0 && r->group[j] < e->k;
                bad = !r->group || r->n_group < 1 || (r->type == SSA_REQ_FORECAST && !any) ||
                      (r->type == SSA_REQ_FORECAST && (r->h < 1 || r->h > SSA_FC_MAX_H));
            }
            if (bad)
            {
                finish_request(s, r, -1);
                keep = 0;
                progressed = 1;
            }
            else if (e->state == RES_READY && u && u->n < s->max_batch && us_reserve(u, u->n + 1) == 0)
            {
                e->refs++;
                lru_unlink(s, e);
                lru_front(s, e);
                u->req[u->n] = r;
                u->res[u->n] = e;
                u->n++;
                keep = 0;
            }
        }
        else if (r->type == SSA_REQ_CADZOW)
        {
            /* a new series: straight to the Cadzow worker */
            const int ok = r->N >= 4 && r->L >= 2 && r->L <= r->N - 1 && r->rank >= 1 && r->max_iter >= 1 &&
                           imin(r->rank, imin(r->L, r->N - r->L + 1)) <= SSA_MAX_KP;
            if (ok)
                cz_push(s, r, NULL, NULL);
            else
                finish_request(s, r, -1);
            keep = 0;
            progressed = 1;
        }
        else if (is_decomp(r))
        {
            if (!r->priv && valid_decomp(s, r))
            {
                /* pending resident entry from the moment the request is seen, so follow-ups on
                 * the series that arrive later wait for it */
                r->priv = res_create(s, r->series_id, r->N, r->L, req_kout(s, r));
                if (!r->priv)
                {
                    s->stats.not_resident++;
                    r->priv = (void *)&g_not_resident;
                }
            }
            if (!valid_decomp(s, r))
            {
                finish_request(s, r, -1);
                keep = 0;
                progressed = 1;
            }
            else if (free_slot && free_slot->n < s->max_batch && (cls < 0 || srv_class(r) == cls))
            {
                cls = srv_class(r);
                const size_t b = ssar_series_bytes(r->N, r->L, r->k, s->p, SRV_GROUPS);
                if (b > s->batch_budget)
                {
                    if (r->priv && r->priv != (void *)&g_not_resident)
                        ((res_entry *)r->priv)->state = RES_FAILED;
                    finish_request(s, r, -1); /* larger than a batch's share of the budget */
                    keep = 0;
                    progressed = 1;
                }
                double *hp[4] = {mapped(r->x), mapped(r->sigma),
                                 r->type == SSA_REQ_DECOMPOSE_RECON ? mapped(r->groups) : NULL,
                                 r->type == SSA_REQ_DECOMPOSE_WCORR ? mapped(r->W) : NULL};
                const int out_direct = (!r->sigma || hp[1]) &&
                                       (r->type != SSA_REQ_DECOMPOSE_RECON || !r->groups || hp[2]) &&
                                       (r->type != SSA_REQ_DECOMPOSE_WCORR || !r->W || hp[3]);
                const size_t in_b = hp[0] ? 0 : (size_t)r->N;
                const size_t nout = req_out_doubles(s, r);
                const size_t out_b = (nout && !out_direct) ? nout : 0;
                if (!keep)
                    ;
                else if (in_b > SRV_STAGE_IN / sizeof(double) || out_b > SRV_STAGE_OUT / sizeof(double))
                {
                    if (r->priv && r->priv != (void *)&g_not_resident)
                        ((res_entry *)r->priv)->state = RES_FAILED;
                    finish_request(s, r, -1); /* pageable buffers larger than the staging area */
                    keep = 0;
                    progressed = 1;
                }
                else if (bytes + b <= s->batch_budget && free_slot->in_used + in_b <= SRV_STAGE_IN / sizeof(double) &&
                         free_slot->out_used + out_b <= SRV_STAGE_OUT / sizeof(double) &&
                         slot_reserve(free_slot, free_slot->n + 1) == 0)
                {
                    slot_t *sl = free_slot;
                    const int j = sl->n;
                    sl->sin[j] = in_b ? sl->in_used : SRV_DIRECT;
                    sl->sout[j] = out_b ? sl->out_used : SRV_DIRECT;
                    memcpy(sl->hp + 4 * (size_t)j, hp, sizeof(hp));
                    sl->in_used += in_b;
                    sl->out_used += out_b;
                    res_entry *e = r->priv == (void *)&g_not_resident ? NULL : (res_entry *)r->priv;
                    if (e && !e->d && res_alloc(s, e) != 0)
                        s->stats.not_resident++; /* runs, but its series will not be resident */
                    sl->req[j] = r;
                    sl->N[j] = r->N;
                    sl->L[j] = r->L;
                    sl->k[j] = r->k;
                    sl->seeds[j] = r->seed;
                    sl->lrf_dst[j] = e ? e->d : NULL;
                    sl->wantw[j] = r->type == SSA_REQ_DECOMPOSE_WCORR;
                    sl->res[j] = e;
                    sl->n++;
                    bytes += b;
                    keep = 0;
                }
            }
        }
        else
        {
            finish_request(s, r, -1);
            keep = 0;
            progressed = 1;
        }
        if (keep)
            s->pend[kept++] = r;
    }
    s->npend = kept;
    if (f && f->n > 0)
    {
        if (fs_launch(s) != 0)
            fs_finish(s, 0);
        progressed = 1;
    }
    if (u && u->n > 0)
    {
        if (us_launch(s) != 0)
            us_finish(s, 0);
        progressed = 1;
    }
    if (free_slot && free_slot->n > 0)
    {
        free_slot->bytes = bytes;
        if (slot_launch(s, free_slot) != 0)
            slot_finish(s, free_slot, 0);
        progressed = 1;
    }
    return progressed;
}

static int any_busy(const ssa_server *s)
{
    if (s->fs.busy || s->us.busy)
        return 1;
    for (int i = 0; i < s->nslots; i++)
        if (s->slots[i].busy)
            return 1;
    return 0;
}

static void *worker(void *arg)
{
    ssa_server *s = (ssa_server *)arg;
    cudaSetDevice(s->device);
    for (;;)
    {
        int progressed = poll_done(s);
        take_queue(s);
        progressed |= dispatch(s);
        if (progressed)
            continue;
        pthread_mutex_lock(&s->mu);
        if (s->stop && s->qcount == 0 && s->npend == 0 && !any_busy(s))
        {
            pthread_mutex_unlock(&s->mu);
            break;
        }
        if (s->qcount == 0)
        {
            if (any_busy(s) || s->npend > 0)
            {
                /* device work in flight (or requests waiting on it): poll again shortly */
                struct timespec ts;
                clock_gettime(CLOCK_REALTIME, &ts);
                ts.tv_nsec += 20000;
                if (ts.tv_nsec >= 1000000000L)
                {
                    ts.tv_sec++;
                    ts.tv_nsec -= 1000000000L;
                }
                pthread_cond_timedwait(&s->cv, &s->mu, &ts);
            }
            else if (!s->stop)
            {
                pthread_cond_wait(&s->cv, &s->mu);
            }
        }
        pthread_mutex_unlock(&s->mu);
    }
    return NULL;
}

/* ---- public API ---------------------------------------------------------------------------- */

int ssa_server_create(ssa_server **out, size_t hbm_budget_bytes, int max_inflight, int max_batch, int oversampling,
                      int power_iters)
{
    if (!out || max_inflight < 1 || max_inflight > 16 || max_batch < 1 || power_iters < 0)
        return -1;
    *out = NULL;
    ssa_server *s = (ssa_server *)calloc(1, sizeof(*s));
    if (!s)
        return -1;
    s->p = oversampling <= 0 ? 8 : oversampling;
    s->q_iters = power_iters;
    s->max_batch = max_batch;
    if (cudaGetDevice(&s->device) != cudaSuccess || ssad_init_device() != 0)
    {
        free(s);
        return -1;
    }
    const int reserve = hbm_budget_bytes != 0;
    if (hbm_budget_bytes == 0)
    {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess)
        {
            free(s);
            return -1;
        }
        hbm_budget_bytes = fr / 10 * 8;
    }
    s->budget = hbm_budget_bytes;
    s->res_budget = hbm_budget_bytes / 4;
    /* device buffers grow by a quarter beyond a batch's estimate: keep the slots inside the budget */
    s->batch_budget = (hbm_budget_bytes - s->res_budget) / (size_t)max_inflight / 5 * 4;
    s->hcap = 65521;
    s->htab = (res_entry **)calloc((size_t)s->hcap, sizeof(res_entry *));
    s->qcap = 1 << 16;
    s->q = (ssa_request **)malloc(sizeof(ssa_request *) * s->qcap);
    s->nslots = max_inflight;
    s->slots = (slot_t *)calloc((size_t)max_inflight, sizeof(slot_t));
    if (!s->htab || !s->q || !s->slots)
    {
        ssa_server_destroy(s);
        return -1;
    }
    pthread_mutex_init(&s->mu, NULL);
    pthread_cond_init(&s->cv, NULL);
    pthread_cond_init(&s->cv_done, NULL);
    for (int i = 0; i < max_inflight; i++)
    {
        slot_t *sl = &s->slots[i];
        if (ssa_rbatch_create(&sl->rb, s->p, power_iters, g_group_idx, g_group_sizes, SRV_GROUPS) != 0 ||
            ssar_set_lrf_group(sl->rb, 2, g_fc_group, 3) != 0 ||
            cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming) != cudaSuccess ||
            ssa_rbatch_set_graphs(sl->rb, 0) != 0 || /* outputs follow each bucket on its stream */
            cudaMallocHost((void **)&sl->h_in, SRV_STAGE_IN) != cudaSuccess ||
            cudaMallocHost((void **)&sl->h_out, SRV_STAGE_OUT) != cudaSuccess ||
            cudaMallocHost((void **)&sl->h_st, sizeof(int) * (size_t)max_batch) != cudaSuccess ||
            cudaMallocHost((void **)&sl->h_lst, sizeof(int) * (size_t)max_batch) != cudaSuccess ||
            !(sl->h_in_d = mapped(sl->h_in)) || !(sl->h_out_d = mapped(sl->h_out)) ||
            cudaMallocHost((void **)&sl->h_seg, sizeof(ssa_copy_seg) * 8 * (size_t)max_batch) != cudaSuccess ||
            !(sl->h_seg_d = (ssa_copy_seg *)mapped(sl->h_seg)) || !(sl->c_seg = 8 * (size_t)max_batch) ||
            (reserve && ssa_rbatch_reserve(sl->rb, s->batch_budget + s->batch_budget / 8) != 0))
        {
            ssa_server_destroy(s);
            return -1;
        }
        for (int r = 0; r < SSAR_NB; r++)
            if (cudaEventCreateWithFlags(&sl->rev[r], cudaEventDisableTiming) != cudaSuccess)
            {
                ssa_server_destroy(s);
                return -1;
            }
    }
    {
        /* forecast batches: tables for max_batch jobs and 4 MB of outputs up front (grown if a
         * batch asks for more) */
        fslot_t *f = &s->fs;
        f->req = (ssa_request **)malloc(sizeof(ssa_request *) * (size_t)max_batch);
        f->res = (res_entry **)malloc(sizeof(res_entry *) * (size_t)max_batch);
        if (!f->req || !f->res || cudaMallocHost((void **)&f->h_jobs, sizeof(ssa_fc_job) * (size_t)max_batch) != cudaSuccess ||
            cudaMalloc((void **)&f->d_jobs, sizeof(ssa_fc_job) * (size_t)max_batch) != cudaSuccess ||
            grow_host((void **)&f->h_out, &f->c_hout, (size_t)1 << 19, sizeof(double)) != 0 ||
            grow_dev((void **)&f->d_out, &f->c_dout, (size_t)1 << 19, sizeof(double)) != 0)
        {
            ssa_server_destroy(s);
            return -1;
        }
        f->cap = max_batch;
    }
    if (reserve)
    {
        /* the resident share of the budget up front: entries are carved from it */
        if (cudaMalloc((void **)&s->res_arena, s->res_budget) != cudaSuccess)
        {
            s->res_arena = NULL;
            ssa_server_destroy(s);
            return -1;
        }
        s->cspans = 1024;
        s->spans = malloc(sizeof(s->spans[0]) * (size_t)s->cspans);
        if (!s->spans)
        {
            ssa_server_destroy(s);
            return -1;
        }
        s->spans[0].off = 0;
        s->spans[0].len = s->res_budget & ~(RA_ALIGN - 1);
        s->nspans = 1;
    }
    {
        /* follow-up batches: one group slot (each series brings its own group) */
        static const int one_idx[1] = {0}, one_size[1] = {1};
        if (ssa_rbatch_create(&s->us.rb, s->p, power_iters, one_idx, one_size, 1) != 0 ||
            cudaEventCreateWithFlags(&s->us.done, cudaEventDisableTiming) != cudaSuccess || us_reserve(&s->us, 64) != 0)
        {
            ssa_server_destroy(s);
            return -1;
        }
    }
    if (cudaStreamCreateWithFlags(&s->fs.st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->fs.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->pool_st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_pool, cudaEventDisableTiming) != cudaSuccess)
    {
        ssa_server_destroy(s);
        return -1;
    }
    pthread_cond_init(&s->cz_cv, NULL);
    if (pthread_create(&s->th, NULL, worker, s) != 0)
    {
        pthread_cond_destroy(&s->cz_cv);
        ssa_server_destroy(s);
        return -1;
    }
    s->th_live = 1;
    if (pthread_create(&s->cz_th, NULL, cz_worker, s) != 0)
    {
        ssa_server_destroy(s);
        return -1;
    }
    s->cz_live = 1;
    *out = s;
    return 0;
}

int ssa_server_submit(ssa_server *s, ssa_request *r)
{
    if (!s || !r)
        return -1;
    r->status = 1; /* in progress */
    r->k_out = 0;
    r->priv = NULL;
    r->iterations = 0;
    r->final_diff = 0.0;
    r->t_done = 0.0;
    r->t_arrival = ssa_server_now();
    pthread_mutex_lock(&s->mu);
    if (s->qcount == s->qcap || s->stop)
    {
        pthread_mutex_unlock(&s->mu);
        r->status = -1;
        return -1;
    }
    s->q[(s->qhead + s->qcount) % s->qcap] = r;
    s->qcount++;
    s->outstanding++;
    s->stats.submitted++;
    pthread_cond_signal(&s->cv);
    pthread_mutex_unlock(&s->mu);
    return 0;
}

int ssa_server_drain(ssa_server *s)
{
    if (!s)
        return -1;
    pthread_mutex_lock(&s->mu);
    while (s->outstanding > 0)
        pthread_cond_wait(&s->cv_done, &s->mu);
    pthread_mutex_unlock(&s->mu);
    return 0;
}

int ssa_server_replay(ssa_server *s, ssa_request *reqs, const double *arrival_s, int n)
{
    if (!s || !reqs || !arrival_s || n < 0)
        return -1;
    const double t0 = ssa_server_now();
    int rc = 0;
    for (int i = 0; i < n; i++)
    {
        const double due = t0 + arrival_s[i];
        for (;;)
        {
            const double now = ssa_server_now();
            if (now >= due)
                break;
            const double d = due - now;
            if (d > 200e-6)
            {
                struct timespec ts = {0, (long)((d - 100e-6) * 1e9)};
                nanosleep(&ts, NULL);
            }
        }
        if (ssa_server_submit(s, &reqs[i]) != 0)
            rc = -1;
    }
    ssa_server_drain(s);
    return rc;
}

int ssa_server_stats_get(ssa_server *s, ssa_server_stats *st)
{
    if (!s || !st)
        return -1;
    pthread_mutex_lock(&s->mu);
    *st = s->stats;
    s->stats.host_launch_max_s = 0.0; /* the maximum is per read */
    st->resident_bytes = s->res_bytes;
    st->resident_budget = s->res_budget;
    st->batch_budget = s->batch_budget;
    pthread_mutex_unlock(&s->mu);
    return 0;
}

void ssa_server_destroy(ssa_server *s)
{
    if (!s)
        return;
    if (s->th_live)
    {
        ssa_server_drain(s);
        pthread_mutex_lock(&s->mu);
        s->stop = 1;
        s->cz_stop = 1;
        pthread_cond_broadcast(&s->cv);
        pthread_cond_broadcast(&s->cz_cv);
        pthread_mutex_unlock(&s->mu);
        pthread_join(s->th, NULL);
        if (s->cz_live)
            pthread_join(s->cz_th, NULL);
        pthread_mutex_destroy(&s->mu);
        pthread_cond_destroy(&s->cv);
        pthread_cond_destroy(&s->cv_done);
        pthread_cond_destroy(&s->cz_cv);
    }
    cudaDeviceSynchronize();
    for (int i = 0; s->slots && i < s->nslots; i++)
    {
        slot_t *sl = &s->slots[i];
        if (sl->rb)
            ssa_rbatch_destroy(sl->rb);
        if (sl->done)
            cudaEventDestroy(sl->done);
        for (int r = 0; r < SSAR_NB; r++)
            if (sl->rev[r])
                cudaEventDestroy(sl->rev[r]);
        void *hp[] = {sl->h_in, sl->h_out, sl->h_st, sl->h_lst, sl->h_seg};
        for (size_t j = 0; j < sizeof(hp) / sizeof(hp[0]); j++)
            if (hp[j])
                cudaFreeHost(hp[j]);
        if (sl->d_x)
            cudaFree(sl->d_x);
        free(sl->req);
        free(sl->N);
        free(sl->L);
        free(sl->k);
        free(sl->seeds);
        free(sl->lrf_dst);
        free(sl->wantw);
        free(sl->res);
        free(sl->xoff);
        free(sl->sin);
        free(sl->sout);
        free(sl->hp);
    }
    free(s->slots);
    if (s->htab)
    {
        while (s->lru_head)
            res_remove(s, s->lru_head);
        free(s->htab);
    }
    if (s->res_arena)
        cudaFree(s->res_arena);
    free(s->spans);
    if (s->pool_st)
    {
        cudaStreamSynchronize(s->pool_st);
        cudaStreamDestroy(s->pool_st);
    }
    if (s->ev_pool)
        cudaEventDestroy(s->ev_pool);
    if (s->fs.st)
        cudaStreamDestroy(s->fs.st);
    if (s->fs.done)
        cudaEventDestroy(s->fs.done);
    if (s->fs.h_jobs)
        cudaFreeHost(s->fs.h_jobs);
    if (s->fs.d_jobs)
        cudaFree(s->fs.d_jobs);
    if (s->fs.h_out)
        cudaFreeHost(s->fs.h_out);
    if (s->fs.d_out)
        cudaFree(s->fs.d_out);
    free(s->fs.req);
    free(s->fs.res);
    {
        uslot_t *u = &s->us;
        if (u->rb)
            ssa_rbatch_destroy(u->rb);
        if (u->done)
            cudaEventDestroy(u->done);
        if (u->h_fc)
            cudaFreeHost(u->h_fc);
        if (u->d_fc)
            cudaFree(u->d_fc);
        if (u->h_out)
            cudaFreeHost(u->h_out);
        if (u->h_lst)
            cudaFreeHost(u->h_lst);
        if (u->d_tmp)
            cudaFree(u->d_tmp);
        if (u->d_fcout)
            cudaFree(u->d_fcout);
        free(u->req);
        free(u->res);
        free(u->N);
        free(u->L);
        free(u->k);
        free(u->goff);
        free(u->gidx);
        free((void *)u->U);
        free((void *)u->V);
        free((void *)u->sig);
        free(u->lrf);
        free(u->tmpoff);
        free(u->hoff);
    }
    free(s->pend);
    free(s->q);
    free(s);
    cudaMemPool_t pool = ssar_pool();
    if (pool)
        cudaMemPoolTrimTo(pool, 0);
}

void *ssa_host_alloc(size_t bytes)
{
    void *p = NULL;
    if (bytes == 0 || cudaMallocHost(&p, bytes) != cudaSuccess)
        return NULL;
    return p;
}

void ssa_host_free(void *p)
{
    if (p)
        cudaFreeHost(p);
}
