/*
 * Request server: continuous batching of decompose / reconstruct / W-correlation / forecast
 * requests of mixed size on one GPU.
 *
 * One worker thread owns the device work. Requests are queued by ssa_server_submit (any thread)
 * and taken in arrival order. Decompositions are gathered into uneven batches (ssa_ragged.c),
 * each batch bounded by a device-memory share of the HBM budget; up to `max_inflight` batches
 * run at once on their own streams, so requests that arrive while others are on the GPU start
 * as soon as a batch slot is free and overlap with the running ones. A decompose+reconstruct
 * request leaves its series resident: the LRF coefficients of the forecast group [0, 1, 2] and
 * the last L - 1 values of that group's reconstruction stay in device memory (stream-ordered
 * pool, least recently used entries evicted beyond the resident share of the budget), so a later
 * forecast request on that series runs the recurrence only (batched, one CTA per request)
 * without decomposing again. Every request is stamped with its arrival and completion times on
 * the host's monotonic clock; completion means its outputs are in host memory.
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
    int refs;          /* in-flight forecasts using it */
    double *d;         /* R (L-1), tail (L-1), verticality */
    size_t bytes;
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

static void res_remove(ssa_server *s, res_entry *e)
{
    res_entry **pp = &s->htab[(unsigned)e->id % (unsigned)s->hcap];
    while (*pp && *pp != e)
        pp = &(*pp)->hnext;
    if (*pp)
        *pp = e->hnext;
    lru_unlink(s, e);
    if (e->d)
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

/* New pending entry for series `id` with window L, without device memory yet (replaces an idle
 * older one); forecasts on the series wait while it is pending. */
static res_entry *res_create(ssa_server *s, int id, int L)
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
    e->state = RES_PENDING;
    unsigned h = (unsigned)id % (unsigned)s->hcap;
    e->hnext = s->htab[h];
    s->htab[h] = e;
    lru_front(s, e);
    return e;
}

/* Device memory for a pending entry when its decomposition is launched: R (L-1), tail (L-1) and
 * verticality doubles, evicting least recently used idle series beyond the resident budget. */
static int res_alloc(ssa_server *s, res_entry *e)
{
    const size_t bytes = sizeof(double) * (2 * (size_t)(e->L - 1) + 1);
    if (res_make_room(s, bytes) != 0)
        return -1;
    cudaMemPool_t pool = ssar_pool();
    if (!pool || cudaMallocFromPoolAsync((void **)&e->d, bytes, pool, s->pool_st) != cudaSuccess)
    {
        e->d = NULL;
        return -1;
    }
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

/* Launch the batch gathered in sl (sl->n requests, dims and staging offsets filled). */
static int slot_launch(ssa_server *s, slot_t *sl)
{
    const double t0 = ssa_server_now();
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
        nseg += req_segs(s, sl->req[i]);
    if (nseg > sl->c_seg)
    {
        if (sl->h_seg)
            cudaFreeHost(sl->h_seg);
        sl->h_seg = sl->h_seg_d = NULL;
        sl->c_seg = 0;
        if (cudaMallocHost((void **)&sl->h_seg, sizeof(ssa_copy_seg) * (nseg + nseg / 2)) != cudaSuccess ||
            !(sl->h_seg_d = (ssa_copy_seg *)mapped(sl->h_seg)))
            return -1;
        sl->c_seg = nseg + nseg / 2;
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
    /* outputs the requests ask for: one scatter launch writing the callers' page-locked buffers,
     * or the staging area slot_finish copies from */
    const size_t *off = ssar_offsets(sl->rb);
    const double *dsig = ssar_sigma(sl->rb), *dW = ssar_W(sl->rb), *dg = ssar_groups(sl->rb);
    for (int i = 0; i < sl->n; i++)
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
    }
    if (ssad_copy_segments(sl->h_seg_d + nin, (int)(ns - nin), ms) != 0)
        return -1;
    if (cudaMemcpyAsync(sl->h_st, ssar_status(sl->rb), sizeof(int) * sl->n, cudaMemcpyDeviceToHost, ms) !=
            cudaSuccess ||
        cudaMemcpyAsync(sl->h_lst, ssar_lrf_status(sl->rb), sizeof(int) * sl->n, cudaMemcpyDeviceToHost, ms) !=
            cudaSuccess ||
        cudaEventRecord(sl->done, ms) != cudaSuccess)
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

static void slot_finish(ssa_server *s, slot_t *sl, int launch_ok)
{
    const double t0 = ssa_server_now();
    for (int i = 0; i < sl->n; i++)
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
        if (e) /* the forecast group [0, 1, 2] needs at least 3 components */
            e->state = (ok && e->d && sl->h_lst[i] == 0 && r->k_out > 2) ? RES_READY : RES_FAILED;
        finish_request(s, r, ok ? 0 : -1);
    }
    sl->n = 0;
    sl->busy = 0;
    sl->in_used = sl->out_used = 0;
    s->stats.host_finish_s += ssa_server_now() - t0;
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

/* ---- worker ---------------------------------------------------------------------------------- */

static int poll_done(ssa_server *s)
{
    int progressed = 0;
    for (int i = 0; i < s->nslots; i++)
    {
        slot_t *sl = &s->slots[i];
        if (!sl->busy)
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
 * length above 32768) take several times longer than the rest, and a batch completes as a whole,
 * so they are batched apart: a short series never waits for a long one's batch. Within a class
 * requests keep their arrival order. */
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
    size_t bytes = 0;
    int kept = 0;
    int cls = -1; /* size class of the batch being formed */
    for (int i = 0; i < s->npend; i++)
    {
        ssa_request *r = s->pend[i];
        int keep = 1;
        if (r->type == SSA_REQ_FORECAST)
        {
            res_entry *e = res_find(s, r->series_id);
            if (!e || e->state == RES_FAILED || r->h < 1 || r->h > SSA_FC_MAX_H)
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
        else if (is_decomp(r))
        {
            if (r->type == SSA_REQ_DECOMPOSE_RECON && !r->priv && valid_decomp(s, r))
            {
                /* pending resident entry from the moment the request is seen, so forecasts on
                 * the series that arrive later wait for it */
                r->priv = res_create(s, r->series_id, r->L);
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
    if (s->fs.busy)
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
    if (cudaStreamCreateWithFlags(&s->fs.st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->fs.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->pool_st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_pool, cudaEventDisableTiming) != cudaSuccess)
    {
        ssa_server_destroy(s);
        return -1;
    }
    if (pthread_create(&s->th, NULL, worker, s) != 0)
    {
        ssa_server_destroy(s);
        return -1;
    }
    s->th_live = 1;
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
        pthread_cond_broadcast(&s->cv);
        pthread_mutex_unlock(&s->mu);
        pthread_join(s->th, NULL);
        pthread_mutex_destroy(&s->mu);
        pthread_cond_destroy(&s->cv);
        pthread_cond_destroy(&s->cv_done);
    }
    cudaDeviceSynchronize();
    for (int i = 0; s->slots && i < s->nslots; i++)
    {
        slot_t *sl = &s->slots[i];
        if (sl->rb)
            ssa_rbatch_destroy(sl->rb);
        if (sl->done)
            cudaEventDestroy(sl->done);
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
