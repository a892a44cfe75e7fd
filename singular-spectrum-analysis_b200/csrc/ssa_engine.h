/*
 * Device pipeline over a set of B series of identical shape (N, L, k + p): the engine that
 * both the reference-compatible single-series API (ssa_api.c, B = 1) and the batched API
 * (ssa_batch.c) drive. Host code in C; all numerics run in ssa_kernels.cu.
 *
 * Per-series device layout (series s):
 *   x64   [s * N]                   input signal (double)
 *   X     [s * ldS]                 signal spectrum, H + 1 complex (ldS floats)
 *   Y     [s * ldL * kp]            L x kp range-finder block (Y, Q, then U in place)
 *   Z     [s * ldK * kp]            K x kp block (Omega, Z, B, then V in place)
 *   recon [s * k * ldN]             k elementary reconstructions (row i = component i)
 * Leading dimensions ldL, ldK, ldN are rounded up to multiples of 4 floats (16 B).
 */
#ifndef SSA_ENGINE_H
#define SSA_ENGINE_H

#include <cuda_runtime_api.h>
#include <stddef.h>
#include <stdint.h>

#include "ssa_kernels.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Kernel kinds for the stage profiler. */
enum
{
    SSAK_SPECTRUM = 0,
    SSAK_CORR,
    SSAK_GRAM,
    SSAK_CHOL,
    SSAK_ROWMUL,
    SSAK_RR,
    SSAK_ELEM,
    SSAK_WFIN,
    SSAK_GSUM,
    SSAK_RECON,
    SSAK_LRF,
    SSAK_WGRAM,                  /* the W-correlation Gram (SSAK_GRAM: the CholQR / Rayleigh-Ritz Grams) */
    SSAK_NKINDS
};
#define SSA_PROF_MAX 512

typedef struct
{
    char *h;    /* pinned host staging */
    char *d;    /* device copy */
    size_t cap;
    size_t used;
    size_t hcap; /* capacity of the pinned block (>= cap when it was recycled) */
} ssa_job_arena;

typedef struct
{
    int B, N, L, K, logh, H, kp, k;
    long long ldL, ldK, ldN, ldS;
    int rows_L, rows_K, rows_N;  /* Gram rows per CTA */
    int nch_L, nch_K, nch_N;     /* Gram partial counts */
    int nq;                      /* rowmul CTAs over L (colsum partials) */
    int device;
    cudaStream_t st;
    int own_stream;
    int recycle;                 /* stream, buffers and pinned arena recycled (own-stream engines) */
    int rowmul_simt;             /* row products on the CUDA cores even when the tensor-core form is on */
    float *Zs;                   /* stacked sweeps: spectra / accumulators of block columns */
    size_t zs_cap;               /* floats */
    float *bsplit;               /* tensor-core row products: split parts of the small factor per series */
    size_t bsplit_cap;           /* series the scratch holds */
    /* device buffers */
    double *x64;
    float *X;
    float *Y, *Z;
    double *part;                /* B * max(nch) * kp(kp+1)/2 */
    double *qsum;                /* B * nq * kp */
    double *Rinv;                /* B * kp * kp: R^{-1} of the last CholQR pass */
    float *Zu, *Zv;              /* B * kp * k */
    double *sigma;               /* B * k */
    int *status;                 /* B */
    float *recon;                /* B * k * ldN (allocated on demand) */
    double *norm2;               /* B * k */
    double *W;                   /* B * k * k */
    float *Us, *Vs;              /* cached spectra B * k * ldS (allocated on demand) */
    /* block power scratch (allocated on demand by ssae_decompose_block) */
    int bcap;                    /* block columns the scratch holds */
    float *Ub, *Vb;              /* B * ldL * 2 bcap, B * ldK * bcap */
    double *xpart;               /* B * max(nch_L, nch_K) * 64 * 64 cross Gram partials */
    float *xC;                   /* B * 64 * 64 deflation coefficients */
    float *sUs, *sVs, *sDinv;    /* B * 64 * 64 small SVD factors */
    int *perm;                   /* B * 64 */
    float *sgn;                  /* B * 64 */
    float *Ut, *Vt;              /* B * ldL * k, B * ldK * k permutation staging */
    ssa_job_arena ja;
    /* SSA_SYNC_CHECK=1 in the environment: wait after every launch and report the first
     * failing stage on stderr (debugging aid; off by default) */
    int sync_check;
    int cur_kind;
    /* stage profiler: event pairs around launches while prof != 0 */
    int prof;
    int nev;
    int ev_kind[SSA_PROF_MAX];
    cudaEvent_t ev[2 * SSA_PROF_MAX];
    double prof_ms[SSAK_NKINDS];
    long long prof_n[SSAK_NKINDS];
} ssa_engine;

/* Enable/disable event timing of every launch (events are created on first use). */
int ssae_set_profiling(ssa_engine *e, int on);
/* Record the start / end of a launch of `kind` (no-op unless profiling). */
void ssae_prof_begin(ssa_engine *e, int kind);
void ssae_prof_end(ssa_engine *e);
/* Wait for the stream, fold recorded intervals into prof_ms / prof_n and reset the list. */
int ssae_prof_collect(ssa_engine *e);

/* Allocate buffers for up to B series. Returns 0 or a cudaError_t value. */
int ssae_create(ssa_engine *e, int B, int N, int L, int kp, int k, cudaStream_t stream);
/* Stream, job arena (arena_bytes) and profiler only, no series buffers: the uneven-batch
 * pipeline (ssa_ragged.c) keeps its own buffers and drives the kernels through this. */
int ssae_create_light(ssa_engine *e, size_t arena_bytes, cudaStream_t stream);
/* Enlarge the job arena to at least `bytes` (waits for the stream first). */
int ssae_grow_arena(ssa_engine *e, size_t bytes);
void ssae_destroy(ssa_engine *e);
/* Device buffers and page-locked blocks of an engine: from the library's stream-ordered pool on
 * the engine's stream and from the recycled page-locked blocks when the engine recycles, else
 * plain cudaMalloc / cudaMallocHost. Return 0 or a cudaError_t value. */
int ssae_dalloc(ssa_engine *e, void **p, size_t bytes);
void ssae_dfree(ssa_engine *e, void *p);
int ssae_pinned(ssa_engine *e, size_t bytes, void **p, size_t *cap);
void ssae_pinned_free(ssa_engine *e, void *p, size_t cap);
/* The library's stream-ordered memory pool on the current device (freed blocks stay cached). */
cudaMemPool_t ssar_pool(void);
int ssae_ensure_recon(ssa_engine *e);
int ssae_ensure_spectra(ssa_engine *e);

/* Pipeline stages (enqueue only; nb <= B series starting at series 0). */
int ssae_signal_spectrum(ssa_engine *e, const double *d_x, int nb);
/* Randomized range finder + Rayleigh-Ritz. d_omega: device K x kp (ld K) per series (stride
 * K * kp), or NULL to generate the test matrix on the device from (seed, series index). */
int ssae_decompose(ssa_engine *e, int nb, int kp, int k, int q, const float *d_omega, long long omega_ld,
                   unsigned long long seed);
int ssae_elem_recon(ssa_engine *e, int nb, int k);
int ssae_wcorr(ssa_engine *e, int nb, int k);
int ssae_spectra(ssa_engine *e, int nb, int k);
/* One correlation sweep on series 0 over `ncols` columns already in Z (forward: Y = H Z) or
 * Y (adjoint: Z = H^T Y). */
int ssae_matvec(ssa_engine *e, int ncols, int adjoint);
/* Block power iteration with Rayleigh-Ritz (reference MKL/ssa_opt.h:1765-1933) for nb
 * series: k components in blocks of bsize, max_iter iterations per block, deflation against the
 * finished components. d_V0: device K x k start blocks per series (stride v0_ld * k, leading
 * dimension v0_ld; block i = columns of that block), or NULL for the device generator. Results
 * in Y (U), Z (V), sigma; sorted by sigma with the reference's sign rule. */
int ssae_decompose_block(ssa_engine *e, int nb, int k, int bsize, int max_iter, const float *d_V0,
                         long long v0_ld, unsigned long long seed);
int ssae_ensure_block(ssa_engine *e, int bcap);
/* Components k_old .. k_new - 1 of series 0 added to the k_old already in Y, Z and sigma by
 * one-column power iterations deflated against them (reference MKL/ssa_opt.h:1935-2056), then
 * all k_new re-sorted by sigma; the sign rule applies to sorted positions >= k_old. */
int ssae_extend(ssa_engine *e, int k_old, int k_new, int max_iter, unsigned long long seed);
/* MSSA randomized decomposition of one instance whose M channels are the engine's first M
 * series (reference MKL/ssa_opt.h:4116-4210, plus q power iterations). d_omega: device K x kp
 * test matrix (ld ldK) or NULL for the generator with `seed`. Results: U_m in Y_m (L x k per
 * channel), V in every Z_m, sigma in series 0's slot. */
int ssae_mssa_decompose(ssa_engine *e, int M, int kp, int k, int q, const float *d_omega, unsigned long long seed);
/* Block power of I stacked operators at once (series i M .. i M + M - 1 are the M channels of
 * instance i): subspace iteration of one block of kp columns from a generated Gaussian start
 * (instance seed: seed ^ golden (i + 1)), q iterations, CholQR of the stacked block after every
 * half step, Rayleigh-Ritz on the last adjoint. Results: U_{i,m} in channel (i, m)'s Y slot,
 * V_i in channel (i, 0)'s Z slot, sigma_i at sigma + i M k, status per instance. */
int ssae_mssa_batch_decompose(ssa_engine *e, int I, int M, int kp, int k, int q, unsigned long long seed);
/* Grouped reconstruction of series s from cached spectra into d_out (double, N). */
int ssae_recon_group(ssa_engine *e, int s, int k, const int *d_group, int n_group, double *d_out);

/* Job arena: copy `sz` bytes of job structs into the staging area, return the device address
 * they will have after ssae_upload_jobs. */
void *ssae_push_jobs(ssa_engine *e, const void *jobs, size_t sz);
int ssae_upload_jobs(ssa_engine *e);
void ssae_reset_jobs(ssa_engine *e);

#ifdef __cplusplus
}
#endif
#endif
