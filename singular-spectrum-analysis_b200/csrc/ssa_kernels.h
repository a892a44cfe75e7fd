/*
 * C-ABI between the C host layer (ssa_host.c) and the sm_100a kernels (ssa_kernels.cu).
 * Plain pointers and sizes only; every pointer is device memory unless its name says host.
 * Each launcher enqueues work on `stream` and returns a cudaError_t value (0 = success)
 * without synchronising.
 *
 * Job tables (arrays of the structs below) live in device memory; one launch processes every
 * job of a table, blockIdx.y selecting the job. Column-major matrices: column c of an m x n
 * matrix with leading dimension ld starts at c * ld. Leading dimensions of float matrices are
 * even, so columns are 8-byte aligned. Spectra are interleaved complex floats (re, im), H + 1
 * values for a real sequence of length M = 2H (bins 0..H).
 */
#ifndef SSA_KERNELS_H
#define SSA_KERNELS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Size limits of the fixed scratch used by ssa_wcorr_noalloc (ssa_b200.h). */
#define SSA_NOALLOC_MAX_N 8192
#define SSA_NOALLOC_MAX_K 32

/* Largest (k + p) the Gram / Cholesky / Rayleigh-Ritz kernels hold on chip. */
#define SSA_MAX_KP 64
/* Rows staged in shared memory per step of the Gram kernel. */
#define SSA_GRAM_CHUNK 128

/* FFT-length bucket: real length M = 2^(logh + 1). */
int ssad_logh_for(int N);
/* FFT size codes of the uneven batches: a logh (4..16, H = 2^logh complex points), or one of the
 * three lengths between the cluster powers of two, H = 3 * 2^13 (real length 49152),
 * H = 5 * 2^13 (81920) and H = 3 * 2^14 (98304), which run on clusters of 3, 5 and 6 CTAs.
 * ssad_spectrum / ssad_corr / ssad_elem_recon1 accept every code. */
#define SSA_FFT_3x13 17
#define SSA_FFT_3x14 18
#define SSA_FFT_5x13 19
#define SSA_FFT_NCODES 20
int ssad_fft_h(int code);       /* complex points H of a size code (0 for an unknown code) */
int ssad_fft_code_for(int N);   /* smallest size code with 2H >= N; -1 beyond N = 131072 */
/* Largest bucket: logh 16 (M = 131072, series up to N = 131072). Buckets up to 14 run one CTA
 * per transform, 15 and 16 a thread-block cluster of 4 or 8 CTAs. */
#define SSA_MAX_LOGH_ALL 16
/* Largest logh one CTA transforms (H = 16384 points, real length 32768). */
#define SSA_ONE_CTA_MAX_LOGH 14

/* Column job for the FFT kernels (signal spectrum, correlation matvec, reconstruction). */
typedef struct
{
    const float *in;      /* column c at in + c * ld_in; NULL => generated N(0,1) (seed) */
    const double *in64;   /* double input (signal spectrum only), used when in == NULL and in64 != NULL */
    const float *in2;     /* second operand column c at in2 + c * ld_in2 (reconstruction: V) */
    float *out;           /* column c at out + c * ld_out */
    const float *X;       /* spectrum of the series (correlation) */
    float *spec;          /* spectrum output (spectrum kernel): column c at spec + c * ld_spec floats */
    const double *scale;  /* optional per-column scale (sigma), NULL = 1 */
    double *norm2;        /* optional per-column weighted norm^2 output (reconstruction) */
    unsigned long long seed;
    long long ld_in, ld_out, ld_spec, ld_in2;
    int n_in, n_out, ncols, n_in2;
    int col0;             /* first generated column index (RNG counter offset) */
    int N, L, K;          /* series dims, used for the diagonal-averaging weights */
    const unsigned long long *seedp; /* device: the generator seed, read at run time (NULL: seed) */
} ssa_col_job;

/* Gram job: part[chunk] = A_chunk^T W A_chunk (n x n, FP64) over rows of A (m x n, ld). */
typedef struct
{
    const float *A;
    double *part;         /* nchunks * n(n+1)/2 doubles: packed upper triangle, row-major */
    double *colsum;       /* optional: nchunks * n partial column sums of A, NULL = skip */
    long long ld;
    int m, n;
    int rows_per_cta;     /* rows folded into one partial (multiple of SSA_GRAM_CHUNK) */
    int weighted;         /* 1: row t weighted by min(t+1, L, K, N-t) */
    int N, L, K;
} ssa_gram_job;

/* Tensor-core W-correlation Gram job: the Gram job plus the series status word (8 = a wait on
 * the tensor cores ran out). */
typedef struct
{
    ssa_gram_job g;
    int *status;
} ssa_wgram_job;

/* Weighted Gram of elementary reconstructions (n <= 64 rows of length m, time-contiguous, the
 * W-correlation input) per chunk of rows_per_cta time steps (a multiple of 32) in the arithmetic
 * ssad_wcorr_tc selects (split-TF32 or split-BF16 products with FP32 accumulation in TMEM, or
 * FP32 on the CUDA cores), FP64 partials in the same packed layout as ssad_gram. */
int ssad_gram_tc(const ssa_wgram_job *d_jobs, int njobs, int maxchunks, void *stream);
/* Which W-correlation Gram the pipelines use: 1 = tensor cores, split TF32 (default); 2 = tensor
 * cores, split BF16; 3 = FP32 products and accumulation per chunk on the CUDA cores (modes 1-3
 * run through ssad_gram_tc's chunked jobs); 0 = FP64 accumulation on the CUDA cores (ssad_gram).
 * The environment variable SSA_WCORR_FP64=1 sets 0 at load. */
void ssad_set_wcorr_tc(int mode);
int ssad_wcorr_tc(void);
/* Time steps per tensor-core W-Gram partial: chunks long enough to amortise a CTA's set-up. */
#define SSA_TC_MIN_ROWS 1024
/* Time steps per W-correlation Gram partial at most (multiple of SSA_GRAM_CHUNK): the partial
 * sums of the tensor-core and FP32 forms accumulate in FP32 within a chunk, and their rounding
 * grows with its length (a batch of few series would otherwise get chunks of thousands of
 * steps). */
#define SSA_W_MAX_ROWS 2048

/* Cholesky job: G = sum of the partials; G = R^T R with R upper triangular; writes R^{-1}
 * (upper triangular, FP64) n x n column-major (X[r][c] at Rinv[r + c n], zeros below the
 * diagonal). */
typedef struct
{
    const double *part;
    double *Rinv;
    int *status;          /* set to a nonzero code on failure (non-finite Gram) */
    int nchunks, n;
    int pad_[2];
} ssa_chol_job;

/* Row products with a small matrix, FP32 accumulation: C[:, 0:p] = A[:, 0:n] * Bm[0:n, 0:p], or
 * sub - A * Bm when sub != NULL. In place allowed (C == A): a CTA reads all columns of its
 * SSA_ROWMUL_ROWS rows before writing them. Bm is FP32 (Bm) or FP64 (Bm64, e.g. R^{-1} of a
 * CholQR pass: Q = Y R^{-1}; rounded to FP32). */
typedef struct
{
    const float *A;
    const float *Bm;      /* n x p col-major, ld = ldb; NULL when Bm64 is given */
    const double *Bm64;   /* n x p col-major, ld = ldb */
    float *C;
    double *colsum;       /* optional: per-CTA partial column sums of C, [blockIdx.x][p] */
    const float *sub;     /* optional: C = sub - A * Bm (sub may alias C), ld = ldsub */
    long long lda, ldc, ldsub;
    int m, n, p, ldb;
    float *Bsplit;        /* tensor-core form: SSA_ROWMUL_BSPLIT_FLOATS of scratch for Bm's split parts */
} ssa_rowmul_job;
/* Scratch floats per job of the tensor-core row products: two phases of 32 inner elements x three
 * TF32 parts x 64 output columns. */
#define SSA_ROWMUL_BSPLIT_FLOATS (2 * 3 * 32 * 64)

/* Cross Gram partials: part[chunk][i * nb + j] = sum over the chunk's rows r of A[r][i] B[r][j]
 * (FP64 accumulation), A m x na (lda), B m x nb (ldb), na, nb <= SSA_MAX_KP. */
typedef struct
{
    const float *A, *B;
    double *part;
    long long lda, ldb;
    int m, na, nb, rows_per_cta;
} ssa_xgram_job;

/* Sum of cross Gram partials into a fp32 na x nb column-major matrix (ld na). */
typedef struct
{
    const double *part;
    float *out;
    int nchunks, na, nb, pad_;
} ssa_xreduce_job;

/* SVD of a small square matrix M = sum of cross Gram partials (n x n, M[i][j] at i * n + j):
 * M = Us diag(sigma) Vs^T by one-sided Jacobi in FP64, sigma descending. Outputs fp32 n x n
 * column-major (ld n): Us, Vs, and Dinv = diag(1 / sigma) (1 where sigma <= 1e-12). */
typedef struct
{
    const double *part;
    double *sigma;
    float *Us, *Vs, *Dinv;
    int *status;
    int nchunks, n;
} ssa_svd_job;

/* Final ordering of a block decomposition: permutation of the k components by sigma (the
 * reference's exchange sort) and signs (sum_i U[i, j] >= 0 after the sort), applied to sigma
 * in place; perm/sign are written for ssa_permcols. */
typedef struct
{
    const float *U;
    double *sigma;
    int *perm;
    float *sign;
    long long ldU;
    int L, k;
    int sign_from; /* the sign rule applies to sorted positions >= sign_from (0: all) */
} ssa_sortsign_job;

/* dst[:, j] = sign[j] * src[:, perm[j]] for j < k, rows < m. */
typedef struct
{
    const float *src;
    float *dst;
    const int *perm;
    const float *sign;
    long long lds, ldd;
    int m, k;
} ssa_permcols_job;

/* Rows of C per k_rowmul CTA (granularity of the colsum partials). */
#define SSA_ROWMUL_ROWS 128

/* Rayleigh-Ritz job: G_B = sum of partials (kp x kp), eigen-decomposition in FP64,
 * sigma (k), Zu = Z[:, :k] and Zv = Z[:, :k] diag(1/sigma), both sign-fixed with the column
 * sums of Q (sum_i U[i, j] >= 0). */
typedef struct
{
    const double *part;
    const double *qsum;   /* nchunks_q * kp partial column sums of Q */
    double *sigma;        /* k */
    float *Zu, *Zv;       /* kp x k, ld = kp */
    int *status;
    int nchunks, nchunks_q, kp, k;
} ssa_rr_job;

/* Reconstruction from cached spectra: out = inv_w * IFFT(sum_{g} Us[g] * Vs[g]). When U is set,
 * the first and last SSA_EDGE anti-diagonals are summed directly from sigma_i U_i and V_i instead
 * (see SSA_EDGE). */
typedef struct
{
    const float *Us, *Vs;     /* spectra: component i at Us + i * ld_spec */
    const int *group;         /* n_group component indices (out of range skipped) */
    double *out64;            /* optional double output (N) */
    float *out;               /* optional float output (N) */
    const float *U, *V;       /* optional factors: column i at U + i * ldU (L rows), V + i * ldV (K rows) */
    const double *sigma;
    long long ld_spec, ldU, ldV;
    int n_group, k;
    int N, L, K;
    int pad_;
} ssa_recon_job;

/* Anti-diagonals at each end of the series that the reconstruction kernels sum directly (FP64)
 * instead of taking from the FP32 FFT convolution: diagonal averaging divides the convolution's
 * roughly uniform absolute rounding error by the anti-diagonal's length, so the short ones at the
 * ends would otherwise dominate the reconstruction error. */
#define SSA_EDGE 128

/* W-correlation finish: W[i][j] = G_ij / sqrt(G_ii G_jj) (0 when a norm <= 1e-12). */
typedef struct
{
    const double *part;
    double *W;                /* k x k row-major */
    int nchunks, k;
} ssa_wfin_job;

/* R-forecast: LRF from U rows (FP64) and the recurrence over the reconstruction. */
typedef struct
{
    const float *U;           /* L x k, ld */
    const int *group;
    const double *recon;      /* N reconstructed values of the group */
    double *R;                /* L - 1 LRF coefficients (output) */
    double *buf;              /* scratch: L - 1 + h */
    double *out;              /* h forecasts */
    double *verticality;
    int *status;
    long long ld;
    int L, N, n_group, h, k;
    int pad_;
} ssa_lrf_job;

/* Group sums of elementary reconstructions: out[s][g][t] = sum_{i in group g} recon[s][i][t]. */
typedef struct
{
    const float *recon;       /* series s, component i at recon + s * recon_series + i * ld_recon */
    long long ld_recon, recon_series;
    const int *group_idx;     /* concatenated component indices */
    const int *group_off;     /* n_groups + 1 offsets into group_idx */
    double *out;              /* series s, group g at out + s * out_series + g * N */
    long long out_series;
    int n_groups, N, k, B;
} ssa_gsum_job;

int ssad_xgram(const ssa_xgram_job *d_jobs, int njobs, int maxchunks, void *stream);
int ssad_xreduce(const ssa_xreduce_job *d_jobs, int njobs, void *stream);
int ssad_svdsmall(const ssa_svd_job *d_jobs, int njobs, void *stream);
int ssad_sortsign(const ssa_sortsign_job *d_jobs, int njobs, void *stream);
int ssad_permcols(const ssa_permcols_job *d_jobs, int njobs, int maxrows, void *stream);
/* out[i] = sum_{s < nslab} in[s * stride + i] for i < n (fixed order; out may alias slab 0). */
int ssad_slabsum(float *out, const float *in, long long stride, int nslab, long long n, void *stream);
/* The same for ninst instances: instance j sums its nslab slabs at in + j * inst_stride into
 * out + j * inst_stride. */
int ssad_slabsum_batch(float *out, const float *in, long long stride, int nslab, long long n, int ninst,
                       long long inst_stride, void *stream);
/* out[s * k + j] = sum_r A[s][r][j]^2 (FP64) for nb column blocks A_s = A + s * sstride (m x k, ld). */
int ssad_colnorm2(const float *A, long long sstride, long long ld, int m, int k, int nb, double *out, void *stream);
/* out2[0] = sum (a - b)^2, out2[1] = sum a^2 over n doubles (FP64, one CTA, fixed order). */
int ssad_diffnorm(const double *a, const double *b, long long n, double *out2, void *stream);
/* The same for nvec vectors of n doubles laid end to end: out2[2 v], out2[2 v + 1]. */
int ssad_diffnorm_batch(const double *a, const double *b, long long n, int nvec, double *out2, void *stream);
/* Segment copies dst[i] = src[i], i < n, one CTA per segment: dst may be page-locked host memory
 * mapped into the device address space, so one launch writes many small outputs straight to the
 * host instead of one copy call each. */
typedef struct
{
    const double *src;
    double *dst;
    long long n;
} ssa_copy_seg;
int ssad_copy_segments(const ssa_copy_seg *d_segs, int nseg, void *stream);
/* x[idx[i]] = recon[idx[i]] for i < n; out2 = {sum (new - old)^2, sum old^2} (gap filling). */
int ssad_gapupdate(double *x, const double *recon, const int *idx, int n, double *out2, void *stream);
/* out[i] = alpha a[i] + beta b[i] (doubles). */
int ssad_axpby(const double *a, const double *b, double *out, double alpha, double beta, long long n, void *stream);
int ssad_init_device(void);
int ssad_group_sum(ssa_gsum_job job, void *stream);
/* Per-series group sums for uneven batches: out[g * N + t] = sum_{i in group g, i < k} recon[i * ld + t]
 * for the series of each job (group index lists shared by all jobs). A job with its own group
 * (gidx != NULL: gn indices) writes that single group to out[t] and ignores the shared lists. */
typedef struct
{
    const float *recon;
    double *out;          /* n_groups x N doubles */
    long long ld_recon;
    int N, k;
    const int *gidx;      /* device, or NULL */
    int gn;
} ssa_rgsum_job;
int ssad_group_sum_ragged(const ssa_rgsum_job *d_jobs, int njobs, int maxN, const int *group_idx,
                          const int *group_off, int n_groups, void *stream);
/* Elementary reconstructions with one FFT buffer: the spectrum of sigma_c u_c is read from
 * spec + c * ld_spec (written by ssad_spectrum), v_c from in2; outputs as ssad_elem_recon. For
 * FFT lengths where two buffers exceed shared memory (logh >= 14). */
int ssad_elem_recon1(const ssa_col_job *d_jobs, int njobs, int maxcols, int logh, void *stream);
/* Largest logh for which ssad_elem_recon (two shared-memory buffers) can run. */
#define SSA_ELEM2_MAX_LOGH 13
int ssad_spectrum(const ssa_col_job *d_jobs, int njobs, int maxcols, int logh, void *stream);
int ssad_corr(const ssa_col_job *d_jobs, int njobs, int maxcols, int logh, void *stream);
/* The correlation of ssad_corr from a precomputed real spectrum of each input column (spec +
 * c ld_spec, H + 1 bins, as ssad_spectrum writes them), single-CTA lengths (logh <= 14): the
 * forward sweep of every channel of a multichannel operator from one transform of the shared
 * block column. With X == NULL the spectrum is taken as the product itself (the inverse step of
 * a stacked adjoint sweep). */
int ssad_corr_spec(const ssa_col_job *d_jobs, int njobs, int maxcols, int logh, void *stream);
/* One channel of a stacked adjoint sweep: forward transform of each input column, conj-product
 * with X, written (first != 0) or added into the column's accumulator at spec + c ld_spec. */
int ssad_corr_acc(const ssa_col_job *d_jobs, int njobs, int maxcols, int logh, int first, void *stream);
/* Correlation sweeps of series of different FFT lengths in one persistent launch: every CTA
 * (512 threads) pops tiles from tiles[0 .. ntiles) through the counter *head (zero before the
 * launch), largest lengths first. A tile is (job, first column c0, logh): the CTA runs the columns
 * c0 .. c0 + 2^(13 - logh) - 1 of that job side by side (those below the job's ncols), each as
 * k_corr does. logh in [SSA_MULTI_MIN_LOGH, SSA_MULTI_MAX_LOGH]. nctas 0: two per SM. */
#define SSA_MULTI_MIN_LOGH 8
#define SSA_MULTI_MAX_LOGH 13
typedef struct
{
    int job, c0, logh, pad_;
} ssa_tile;
int ssad_corr_multi(const ssa_col_job *d_jobs, const ssa_tile *d_tiles, int ntiles, int *d_head, int nctas,
                    void *stream);
/* The sweep of ssad_corr over a column list of tiles (job, column c0; logh unused): one CTA
 * (cluster) per tile, so that no CTA is spent on columns beyond a job's ncols. */
int ssad_corr_tiles(const ssa_col_job *d_jobs, const ssa_tile *d_tiles, int ntiles, int logh, void *stream);
/* Columns one tile of the multi-length sweep covers at logh. */
int ssad_multi_tile_cols(int logh);
int ssad_elem_recon(const ssa_col_job *d_jobs, int njobs, int maxcols, int logh, void *stream);
/* All jobs of one launch share `weighted`. */
int ssad_gram(const ssa_gram_job *d_jobs, int njobs, int maxchunks, int weighted, void *stream);
int ssad_chol(const ssa_chol_job *d_jobs, int njobs, void *stream);
int ssad_rowmul(const ssa_rowmul_job *d_jobs, int njobs, int maxrows, int maxn, void *stream);
/* The same products on the 5th-generation tensor cores: both operands split into three TF32
 * parts, the six part products down to 2^-22 relative accumulated in FP32 in TMEM (FP32-level
 * rounding). ssad_rowmul_tc_on() says whether the randomized pipelines use it (default 0;
 * block power always keeps the CUDA-core form). */
int ssad_rowmul_tc(const ssa_rowmul_job *d_jobs, int njobs, int maxrows, int maxn, void *stream);
void ssad_set_rowmul_tc(int on);
int ssad_rowmul_tc_on(void);
int ssad_rr(const ssa_rr_job *d_jobs, int njobs, void *stream);
int ssad_recon(const ssa_recon_job *d_jobs, int njobs, int logh, void *stream);
int ssad_wfin(const ssa_wfin_job *d_jobs, int njobs, void *stream);
int ssad_lrf(const ssa_lrf_job *d_jobs, int njobs, void *stream);
/* R-forecast from stored LRF coefficients: out[t] = sum_{j < w} R[j] v[t + j] for t < h, where
 * v = (tail[0..w), out[0..t)) (the recurrence of MKL/ssa_opt.h:2818-2841). One CTA per job. */
typedef struct
{
    const double *R;      /* w = L - 1 coefficients */
    const double *tail;   /* last w reconstructed values */
    double *out;          /* h forecasts */
    int w, h;
} ssa_fc_job;
#define SSA_FC_MAX_H 4096
int ssad_forecast_apply(const ssa_fc_job *d_jobs, int njobs, void *stream);
/* Column-major K x ncols N(0,1) matrix from the device generator (the same values the
 * correlation kernel generates when its input is NULL). */
int ssad_gaussian(float *out, long long ld, int rows, int ncols, int col0, unsigned long long seed,
                  void *stream);
/* Read (and optionally reset) the device self-check record {violations, kernel, block, code,
 * value} of the current device. */
int ssad_read_checks(unsigned int *out5, int reset);
/* Real FFT length 32768 on 2-CTA clusters of 8192-point CTAs (on != 0) or one CTA of 1024
 * threads per transform (0, the default). */
void ssad_set_cl14(int on);
int ssad_cl14(void);
/* Add n kernel launches to the count (a CUDA-graph replay launches the kernels it captured). */
void ssad_count_launches(unsigned long long n);
/* Count of kernel launches issued by this library since load (all devices). */
unsigned long long ssad_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
