/*
 * ssa_b200.h — additions of the B200 SSA library beyond the reference interface.
 * Included by ssa_opt.h. None of these functions changes the behaviour of a reference entry
 * point; they add what the reference API cannot express.
 */
#ifndef SSA_B200_H
#define SSA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Randomized decomposition with `power_iters` subspace iterations and an optional
 * caller-supplied Gaussian test matrix Omega (K x kp, column-major, kp = min(k + p, L, K)).
 * Omega == NULL draws the matrix from the library generator like
 * ssa_opt_decompose_randomized. power_iters == 0 with the same Omega is the reference
 * algorithm of MKL/ssa_opt.h:1685-1763 (ssa_opt_decompose_randomized). Requires
 * ssa_opt_prepare. Returns 0 or -1. */
int ssa_opt_decompose_randomized_ex(SSA_Opt *ssa, int k, int oversampling, int power_iters, const double *Omega);

/* Block power decomposition (reference: ssa_opt_decompose_block, MKL/ssa_opt.h:1765-1933)
 * with caller-supplied start blocks V0 (K x k column-major; the columns of block i start block
 * i), or V0 == NULL for the library generator. Returns 0 or -1. */
int ssa_opt_decompose_block_ex(SSA_Opt *ssa, int k, int block_size, int max_iter, const double *V0);

/* MSSA analogue of ssa_opt_decompose_randomized_ex (reference: mssa_opt_decompose,
 * MKL/ssa_opt.h:4116-4210). */
int mssa_opt_decompose_ex(MSSA_Opt *mssa, int k, int oversampling, int power_iters, const double *Omega);

/* ---- batched pipeline ---------------------------------------------------------------------
 * One launch sequence runs the whole hot path for up to max_series series of identical
 * (N, L): randomized decomposition (k, oversampling, power_iters), every elementary
 * reconstruction, the W-correlation matrix and the sums of the requested component groups. */
typedef struct ssa_batch ssa_batch;

/* groups: n_groups groups, group g has group_sizes[g] indices listed consecutively in
 * group_idx. Returns 0 or -1. */
int ssa_batch_create(ssa_batch **out, int max_series, int N, int L, int k, int oversampling, int power_iters,
                     const int *group_idx, const int *group_sizes, int n_groups);
void ssa_batch_destroy(ssa_batch *b);

/* Device-resident run: d_x is B x N doubles (row s = series s) in device memory. Results stay
 * on the device (ssa_batch_device_results). Enqueues on the batch stream and returns without
 * waiting; seed selects the test matrices (series s uses stream (seed, s)). */
int ssa_batch_run_device(ssa_batch *b, const double *d_x, int B, uint64_t seed);

/* Host-to-host run through the same pipeline: x is B x N doubles; outputs (host, any may be
 * NULL): sigma B x k, W B x k x k (row-major per series), groups B x n_groups x N. Waits for
 * completion. Returns 0, or -1 when any series failed. */
int ssa_batch_run(ssa_batch *b, const double *x, int B, uint64_t seed, double *sigma, double *W,
                  double *groups);

/* Device pointers to the results of the last run (strides in elements). */
typedef struct
{
    const double *sigma;      /* B x k */
    const double *W;          /* B x k x k */
    const double *groups;     /* B x n_groups x N */
    const float *recon;       /* elementary reconstructions: series s, component i at
                                 recon + (s * k + i) * ld_recon */
    long long ld_recon;
    const int *status;        /* B status words (0 = ok) */
    void *stream;             /* cudaStream_t of the batch */
} ssa_batch_results;

int ssa_batch_device_results(const ssa_batch *b, ssa_batch_results *out);
/* Copy the status words of the first n series of the last run (0 = ok; bit 0: non-finite
 * Gram in an orthonormalisation, bit 1: non-finite Rayleigh-Ritz result). Waits for the batch
 * stream. Returns 0 or -1. */
int ssa_batch_status(ssa_batch *b, int *status, int n);
/* Wait for the batch stream; returns 0 when every series of the last run succeeded. */
int ssa_batch_sync(ssa_batch *b);

/* The Hankel matvecs of the context (the reference's static ssa_opt_hankel_matvec /
 * ssa_opt_hankel_matvec_T, MKL/ssa_opt.h:871-903): y = H v (v: K values, y: L values) and
 * z = H^T u (u: L values, z: K values), host arrays, computed on the device in FP32. */
int ssa_opt_hankel_matvec_dev(SSA_Opt *ssa, const double *v, double *y);
int ssa_opt_hankel_matvec_T_dev(SSA_Opt *ssa, const double *u, double *z);

/* Copy the host factor arrays of a decomposed context: U (L x k) and V (K x k), column-major,
 * k = n_components. Either pointer may be NULL. Returns k or -1. */
int ssa_opt_copy_factors(const SSA_Opt *ssa, double *U, double *V);

/* The same for a decomposed MSSA context: U ((M L) x k, channel m in rows m L .. m L + L - 1),
 * V (K x k) and sigma (k). Any pointer may be NULL. Returns k or -1. */
int mssa_opt_copy_factors(const MSSA_Opt *mssa, double *U, double *V, double *sigma);

/* Arithmetic of the W-correlation Gram in every pipeline (single series, batches, server):
 * 1 (default) = 5th-generation tensor cores, split-TF32 products (hi hi^T + lo hi^T + hi lo^T)
 * with FP32 accumulation in TMEM per chunk of >= 1024 time steps and FP64 across chunks;
 * 0 = FP64 accumulation of FP32 products on the CUDA cores. SSA_WCORR_FP64=1 in the environment
 * selects 0 at start-up. No counterpart in the reference (its W-correlation is FP64 dsyrk). */
void ssa_b200_set_wcorr_tensor_cores(int on);
int ssa_b200_wcorr_tensor_cores(void);
/* The W-correlation Gram's arithmetic in full: SSA_WGRAM_FP64 (0) FP64 accumulation of FP32
 * products on the CUDA cores; SSA_WGRAM_TF32X3 (1, the default) tensor cores, split TF32 as
 * above; SSA_WGRAM_BF16X3 (2) tensor cores, split BF16 (hi, lo of 8 significant bits each, the
 * same three products; ~16-bit products, for comparison); SSA_WGRAM_FP32 (3) FP32 products
 * accumulated in FP32 per chunk of >= 1024 time steps on the CUDA cores, FP64 across chunks.
 * Returns 0, or -1 for another mode. */
enum
{
    SSA_WGRAM_FP64 = 0,
    SSA_WGRAM_TF32X3 = 1,
    SSA_WGRAM_BF16X3 = 2,
    SSA_WGRAM_FP32 = 3
};
int ssa_b200_set_wcorr_gram(int mode);
int ssa_b200_wcorr_gram(void);
/* Row products of the randomized pipelines (Q = Y R^{-1} of every CholQR pass, U = Q Z_u,
 * V = B Z_v; single series, batches, MSSA, the server) on the tensor cores (1): both operands
 * split into three TF32 parts and the six part products down to 2^-22 relative accumulated in
 * FP32 in TMEM, i.e. FP32-level rounding (results within ~1e-7 of the CUDA-core form); 0 (the
 * default, faster on the mixed stream) = FP32 on the CUDA cores. Block power (decompose_block,
 * extend, the multichannel batch) always uses the CUDA-core form. SSA_ROWMUL_TC=1 in the
 * environment selects 1 at start-up. */
void ssa_b200_set_rowmul_tensor_cores(int on);
int ssa_b200_rowmul_tensor_cores(void);

/* Context recycling (default on): contexts that own their stream (SSA_Opt, MSSA_Opt, uniform
 * and multichannel batches) take the stream from a per-device stack that freed contexts return
 * it to, their device buffers from the library's stream-ordered memory pool (freed blocks stay
 * cached), and their page-locked staging from a per-device free list, so that creating and
 * freeing a context per series costs no device-wide synchronisation or page pinning. 0 restores
 * plain cudaMalloc / cudaMallocHost / stream creation for contexts created afterwards. No
 * counterpart in the reference (a CPU library). */
void ssa_b200_set_context_recycling(int on);
int ssa_b200_context_recycling(void);

/* ---- Uneven batches ------------------------------------------------------------------------
 * B series of different lengths N[s], windows L[s] and ranks k[s] (common oversampling p and
 * power iterations q) through the same pipeline as ssa_batch_*: randomized decomposition with
 * the device generator (series s seeded seed ^ 0x9E3779B97F4A7C15 (s + 1), as in ssa_batch_*),
 * all k[s] elementary reconstructions, W-correlation and group sums. Series are bucketed by FFT
 * length (N <= 131072); each bucket runs one launch per
 * stage on its own stream and the buckets overlap on the device. (M is the FFT length
 * ssa_b200_fft_length(N): a power of two or one of the mixed lengths 49152 / 81920 / 98304.) No
 * counterpart in the reference, whose API takes one series per context.
 *
 * Inputs and outputs are packed in series order: x holds N[s] doubles at sum_{t<s} N[t];
 * sigma k'[s] at sum_{t<s} k'[t]; W k'[s]^2 (row-major) at sum_{t<s} k'[t]^2; groups
 * n_groups x N[s] at n_groups sum_{t<s} N[t], where k'[s] = min(k[s], L[s], N[s] - L[s] + 1).
 * ssa_rbatch_layout returns these offsets (4 per series: x, sigma, W, groups) and the four
 * totals of the last run. Device buffers grow as needed and are reused across runs.
 * Returns 0 / -1 (invalid shape, N > 131072, k + p > 64, or a series whose decomposition
 * failed). */
typedef struct ssa_rbatch ssa_rbatch;
int ssa_rbatch_create(ssa_rbatch **out, int oversampling, int power_iters, const int *group_idx,
                      const int *group_sizes, int n_groups);
void ssa_rbatch_destroy(ssa_rbatch *b);
int ssa_rbatch_run(ssa_rbatch *b, int B, const int *N, const int *L, const int *k, const double *x,
                   uint64_t seed, double *sigma, double *W, double *groups);
/* d_x in device memory; enqueues only (ssa_rbatch_sync waits and checks every series). */
int ssa_rbatch_run_device(ssa_rbatch *b, int B, const int *N, const int *L, const int *k, const double *d_x,
                          uint64_t seed);
/* The same runs with per-series outputs: want_w[i] = 1 computes the W-correlation of series i
 * (and all k elementary reconstructions it needs); 0 skips it, computes only the elementary
 * reconstructions of the components the groups name, and leaves that series' W block zero.
 * want_w == NULL is the plain run (W for every series). A request that only asks for grouped
 * reconstructions (the reference's decompose + reconstruct) then costs no W-correlation work. */
int ssa_rbatch_run_ex(ssa_rbatch *b, int B, const int *N, const int *L, const int *k, const double *x,
                      uint64_t seed, double *sigma, double *W, double *groups, const unsigned char *want_w);
int ssa_rbatch_run_device_ex(ssa_rbatch *b, int B, const int *N, const int *L, const int *k, const double *d_x,
                             uint64_t seed, const unsigned char *want_w);
int ssa_rbatch_sync(ssa_rbatch *b);
/* Series whose transforms fit one CTA of 512 threads (real FFT lengths 512 .. 16384) share one
 * bucket whose correlation sweeps are one persistent launch: every CTA pops (series, column
 * group, length) tiles from a work queue in device memory, longest lengths first, and runs the
 * columns of shorter lengths side by side. Off (0), every FFT length is a bucket of its own with
 * one launch per stage. On by default. No counterpart in the reference. */
void ssa_b200_set_multi_length(int on);
int ssa_b200_multi_length(void);
/* Launch parameters of the uneven batches chosen per FFT-length bucket (the autotuner of
 * ssa_tune.py measures candidates and sets them; 0 keeps the built-in heuristic):
 * gram_ctas[code] the CTA count the Gram partial launches of the bucket with size code `code`
 * aim at (n entries, codes as ssa_b200_fft_size_code), multi_ctas_per_sm the CTAs per SM of the
 * persistent multi-length sweep (1 or 2). Host state of the process; returns 0 / -1. get returns
 * the number of size codes. No counterpart in the reference. */
int ssa_b200_tune_set(const int *gram_ctas, int n, int multi_ctas_per_sm);
int ssa_b200_tune_get(int *gram_ctas, int n, int *multi_ctas_per_sm);
/* Transforms of real length 32768 (series of 16385 <= N <= 32768) on thread-block clusters of
 * two 8192-point CTAs exchanging through distributed shared memory (on != 0) or on one CTA of 1024
 * threads each (0, the default): a per-bucket choice of the autotuner. The same values either way
 * up to FP32 rounding. */
void ssa_b200_set_cluster32k(int on);
int ssa_b200_cluster32k(void);
/* Size code of the FFT length for a series of length N (the bucket index the tuning table uses):
 * log2 of the complex length for powers of two, other values for the mixed lengths; -1 beyond
 * N = 131072. */
int ssa_b200_fft_size_code(int N);
/* Real FFT length an uneven batch (and the server) uses for a series of length N: the smallest
 * of 2^a (a <= 17), 49152, 81920 and 98304 that is >= N (at least 32), or -1 beyond N = 131072. The
 * single-series API and the uniform batch use the power of two. No counterpart in the reference
 * (whose FFT length is the power of two >= N + K - 1). */
int ssa_b200_fft_length(int N);
/* Every buffer of a run lives in one device arena, grown in stream order when a run needs more;
 * reserving it up front keeps growth (and the driver allocation behind it) out of later runs. */
int ssa_rbatch_reserve(ssa_rbatch *b, size_t bytes);
int ssa_rbatch_layout(const ssa_rbatch *b, size_t *offsets, size_t *totals);
/* Device pointers of the packed outputs and the stream every run ends on (recon is NULL). */
int ssa_rbatch_device_results(const ssa_rbatch *b, ssa_batch_results *out);
/* Outputs of series s of the last run, copied to host arrays after waiting for the run: sigma
 * (k'), W (k' x k', zero unless computed), groups (n_groups x N), and the factors U (L x k') and
 * V (K x k', column-major, FP32 on the device, widened). Any pointer may be NULL. Returns k' or
 * -1. */
int ssa_rbatch_series_result(ssa_rbatch *b, int s, double *sigma, double *W, double *groups, double *U,
                             double *V);
/* on: 0 off, 1 per-kernel CUDA-event times (buckets overlap, so the intervals include other
 * buckets' work), 2 the same with the buckets run one after another (isolated launch times). */
int ssa_rbatch_set_profiling(ssa_rbatch *b, int on);
int ssa_rbatch_profile(ssa_rbatch *b, double *ms, long long *launches, int nkinds);
/* CUDA graphs of whole runs (on by default): when a run has the launch signature of the previous
 * run (the same shapes, per-series options, input and buffer addresses; the generator seed may
 * differ, it is read from device memory) the run is captured as one graph of all buckets'
 * launches and copies, and later runs with that signature replay it after restoring the job
 * tables into the staging areas: one launch call instead of one per stage per bucket. Up to four
 * graphs per batch, least recently used replaced. Profiling runs never use graphs. */
int ssa_rbatch_set_graphs(ssa_rbatch *b, int on);
int ssa_rbatch_graph_stats(const ssa_rbatch *b, long long *captures, long long *replays);

/* ---- Batched multichannel SSA with Cadzow iterations --------------------------------------------
 * I independent instances of M channels of length N each (the stacked (M L) x K trajectory
 * operator of MKL/ssa_opt.h:3880-4283 per instance), all processed together, and `iters`
 * multivariate Cadzow iterations (the reference's ssa_opt_cadzow loop, MKL/ssa_opt.h:3165-3290,
 * applied to the stacked operator: rank-k projection, then every channel replaced by its
 * reconstruction from the k components). Each projection is a block power decomposition of the
 * instance's stacked operator: one block of kp = min(k + p, M L, K) columns from the device
 * generator (instance seed: seed ^ 0x9E3779B97F4A7C15 (i + 1), the same every iteration),
 * power_iters subspace iterations with CholQR of the stacked block after every half step, and a
 * Rayleigh-Ritz step. Channel data is instance-major: channel m of instance i at (i M + m) N.
 * No counterpart in the reference (whose MSSA is randomized only and whose Cadzow is one channel).
 * Returns 0 / -1. */
typedef struct ssa_mbatch ssa_mbatch;
int ssa_mbatch_create(ssa_mbatch **out, int I, int M, int N, int L, int k, int oversampling, int power_iters);
void ssa_mbatch_destroy(ssa_mbatch *b);
/* Device input d_X (I M N doubles); enqueues only. d_out: the channels after the iterations (I M
 * N), d_sigma: each instance's k singular values of the last projection (I x k); either may be
 * NULL. */
int ssa_mbatch_run_device(ssa_mbatch *b, const double *d_X, int iters, uint64_t seed, double *d_out,
                          double *d_sigma);
/* Waits for the run; 0 when every instance's decompositions succeeded. */
int ssa_mbatch_sync(ssa_mbatch *b);
/* Relative change of every iteration: diff[i iters + t] = ||y_t - y_{t-1}|| / ||x|| over the M
 * channels of instance i (y_{-1} = x). Waits for the run. */
int ssa_mbatch_diffs(ssa_mbatch *b, int iters, double *diff);
/* Host-to-host run (out, sigma, diff as above, host arrays, any may be NULL). */
int ssa_mbatch_run(ssa_mbatch *b, const double *X, int iters, uint64_t seed, double *out, double *sigma,
                   double *diff);
/* Components k and block columns kp the batch computes; its stream. */
int ssa_mbatch_dims(const ssa_mbatch *b, int *k, int *kp);
void *ssa_mbatch_stream(const ssa_mbatch *b);

/* ---- Request server ------------------------------------------------------------------------
 * Continuous batching of mixed-size requests on one GPU (no counterpart in the reference, whose
 * API is one synchronous call per series). A worker thread takes submitted requests in arrival
 * order and gathers decompositions into uneven batches (ssa_rbatch_*), each within a share of
 * the device-memory budget; up to max_inflight batches run at once on their own streams, so
 * requests that arrive while others are on the GPU start as soon as a batch slot and memory are
 * free. Decompositions use the randomized pipeline with oversampling p and q power iterations,
 * the device generator seeded with the request's `seed`, and compute the reconstructions of
 * groups [0] and [1, 2] and the W-correlation matrix.
 *
 * A decomposition request leaves its series resident under series_id: its factors U, V and sigma
 * (FP32 / FP64), its signal, and the LRF coefficients of the group [0, 1, 2]
 * (MKL/ssa_opt.h:2766-2816) with the last L - 1 values of that group's reconstruction stay in
 * device memory, a quarter of the budget at most (least recently used series evicted first).
 * Follow-up requests on a resident series do not decompose again:
 *   SSA_REQ_FORECAST      h-step R-forecast (:2818-2867) of `group` (NULL: [0, 1, 2], whose LRF
 *                         and tail are already resident, so only the recurrence runs);
 *   SSA_REQ_RECONSTRUCT   reconstruction of `group` (:2325-2400) into out (N values);
 *   SSA_REQ_CADZOW        with x == NULL: Cadzow iterations (:3165-3290) of rank `rank` on the
 *                         resident signal, the first projection taken from the resident factors
 *                         (rank <= k'), the later ones decomposing as the reference does; with x
 *                         given (and N, L): the same on a new series. Output in out (N values),
 *                         iterations and final_diff set.
 * Reconstructions and group forecasts of resident series run in batches of their own (one
 * launch per stage per FFT-length bucket, elementary reconstructions of the resident factors);
 * Cadzow requests run one after another on a worker of their own, overlapping the batches. A
 * follow-up that arrives while its series' decomposition is still queued or running waits for
 * it. Requests fail (status -1) on invalid shapes, N > 131072, k + p > 64, a series larger than
 * a batch's share of the budget, a follow-up on a series that is not resident, an empty group,
 * an LRF whose verticality coefficient is >= 1, or a forecast group with no component below k'.
 * Output pointers may be NULL; they must stay valid until the request completes. */
enum
{
    SSA_REQ_DECOMPOSE_RECON = 0, /* outputs: sigma, groups (2 x N: [0] then [1, 2]) */
    SSA_REQ_DECOMPOSE_WCORR = 1, /* outputs: sigma, W (k' x k', row-major) */
    SSA_REQ_FORECAST = 2,        /* outputs: forecast (h values after the series' end) */
    SSA_REQ_RECONSTRUCT = 3,     /* outputs: out (N values) */
    SSA_REQ_CADZOW = 4           /* outputs: out (N values), iterations, final_diff */
};
typedef struct
{
    int type;
    int series_id;      /* resident key (decompositions) or target (follow-ups) */
    int N, L, k;        /* decompositions (and Cadzow on a new series: N, L) */
    int h;              /* forecast steps (1 .. 4096) */
    const double *x;    /* decompositions: N input values (host); Cadzow: NULL = resident signal */
    uint64_t seed;      /* generator seed of the decomposition */
    double *sigma;      /* k' = min(k, L, N - L + 1) values */
    double *groups;     /* 2 x N */
    double *W;          /* k' x k' */
    double *forecast;   /* h */
    /* set by the server */
    int status;         /* 1 while in progress, then 0 (done) or -1 (failed) */
    int k_out;          /* k' */
    double t_arrival;   /* seconds on ssa_server_now's clock */
    double t_done;
    void *priv;         /* reserved for the server */
    /* follow-ups and Cadzow */
    const int *group;   /* component indices (host), n_group of them; NULL: the type's default */
    int n_group;
    int rank;           /* Cadzow rank */
    int max_iter;       /* Cadzow iterations at most */
    double tol;         /* Cadzow stopping threshold on the relative change */
    double *out;        /* RECONSTRUCT / CADZOW: N values */
    int iterations;     /* set by the server (Cadzow) */
    double final_diff;  /* set by the server (Cadzow) */
} ssa_request;
typedef struct
{
    long long submitted, completed, failed;
    long long batches, decompositions, max_batch;
    long long forecast_batches, forecasts;
    long long evictions, not_resident;
    size_t resident_bytes, resident_budget, batch_budget;
    double host_launch_s, host_finish_s; /* worker time spent forming / completing batches */
    double host_launch_max_s;            /* longest forming of one batch since the previous read */
    long long followup_batches, followups; /* reconstruction / group-forecast batches on resident factors */
    long long cadzow_requests, cadzow_iterations;
} ssa_server_stats;
typedef struct ssa_server ssa_server;
/* hbm_budget_bytes 0: 80 % of the free device memory at creation, device memory taken as batches
 * need it; an explicit budget reserves every batch slot's device arena at creation. */
int ssa_server_create(ssa_server **out, size_t hbm_budget_bytes, int max_inflight, int max_batch, int oversampling,
                      int power_iters);
/* Waits for every submitted request, then stops the worker and frees everything. */
void ssa_server_destroy(ssa_server *s);
/* Thread-safe; stamps t_arrival. The request must stay valid until it completes. */
int ssa_server_submit(ssa_server *s, ssa_request *r);
/* Wait until every submitted request has completed. */
int ssa_server_drain(ssa_server *s);
/* Submit reqs[i] at arrival_s[i] seconds after the call (ascending), then drain. */
int ssa_server_replay(ssa_server *s, ssa_request *reqs, const double *arrival_s, int n);
int ssa_server_stats_get(ssa_server *s, ssa_server_stats *st);
double ssa_server_now(void);
/* Page-locked host memory. Request inputs and outputs in page-locked memory are copied straight
 * to and from the device; pageable ones go through a fixed staging area per batch slot (256 MB in,
 * 512 MB out), which bounds how many of them one batch takes (a request whose pageable buffers
 * alone exceed it fails). All output buffers of one request should be of the same kind. */
void *ssa_host_alloc(size_t bytes);
void ssa_host_free(void *p);

/* Stage profiler of a batch: with profiling on, every kernel launch of ssa_batch_run* is
 * bracketed by CUDA events on the batch stream. ssa_batch_profile waits for the stream and
 * returns the accumulated milliseconds and launch counts per kernel kind in the order
 * spectrum, corr, gram, chol, rowmul, rr, elem_recon, wcorr_finish, group_sum, recon, lrf.
 * Returns the number of kinds (11) or -1. */
int ssa_batch_set_profiling(ssa_batch *b, int on);
int ssa_batch_profile(ssa_batch *b, double *ms, long long *launches, int nkinds);

/* ---- W-correlation without device allocation --------------------------------------------
 * No counterpart in the reference: an addition for callers that must not have device memory
 * allocated on their behalf, such as a host application whose device memory is owned up
 * front by another framework's allocator, or a latency-critical loop that cannot take the
 * implicit device synchronisation of cudaMalloc. It computes the k x k W-correlation matrix
 * (row-major, FP64) of a decomposition the caller already holds in device memory: U (L x k,
 * column-major, leading dimension ldU), V (K x k, ldV), sigma (k doubles), K = N - L + 1, and
 * writes it to the device array d_W. It calls no cudaMalloc, cudaFree or other allocating
 * routine: its scratch is one fixed array of about 1.1 MB inside the library, which every GPU
 * that loads the library holds until the process exits. Limits: N <= 8192 and k <= 32
 * (larger sizes return -2 without touching the GPU); ldU and ldV even and U, V 8-byte aligned.
 * The work is enqueued on `stream` (a cudaStream_t, NULL for the default stream) and the call
 * returns without waiting (its job tables travel as kernel parameters). The first call on a
 * device also performs that device's one-time set-up (the library's twiddle table upload, if no
 * other entry point did it yet, and the lookup of the scratch array's device address), so make
 * the first call on each device before any stream capture. That set-up is kept for the process:
 * calls must not span a cudaDeviceReset of the device. All calls on a device share the
 * scratch array, which keeps the previous call's contents: calls that may overlap on the GPU
 * (different streams without ordering between them) race and must be serialised by the
 * caller. Returns 0, -1 (invalid argument or CUDA error) or -2 (size beyond the limits). */
int ssa_wcorr_noalloc(const float *d_U, long long ldU, const float *d_V, long long ldV, const double *d_sigma,
                      int N, int L, int k, double *d_W, void *stream);

/* ---- library information ------------------------------------------------------------------ */
/* Number of CUDA kernel launches issued by this library in this process. */
unsigned long long ssa_b200_kernel_launches(void);
/* Eigenvalues (wr + i wi) of a real n x n row-major matrix: the host solver ssa_opt_parestimate
 * uses (Householder-Hessenberg reduction and Francis double-shift QR, FP64), exported so that it
 * can be checked on its own. No counterpart in the reference (which calls LAPACK dgeev). 0 / -1. */
int ssa_b200_eigvals(int n, const double *A, double *wr, double *wi);
/* Device self-check record of the current device: {violations, kernel, block, code, value};
 * kernels that validate their job tables record the first violation there instead of
 * accessing memory with it. reset != 0 clears the record. Returns 0 or -1. */
int ssa_b200_device_checks(unsigned int *out5, int reset);
/* sizeof(SSA_Opt) as compiled into the library. */
int ssa_b200_sizeof_ssa_opt(void);

#ifdef __cplusplus
}
#endif
#endif
