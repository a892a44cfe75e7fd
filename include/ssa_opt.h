/*
 * ssa_opt.h — drop-in C API of the B200 SSA library (libssa.so).
 *
 * Replaces the public interface of SSA-Opt's MKL/ssa_opt.h (declarations at
 * MKL/ssa_opt.h:318-430, structs at :145-315, :374-413) and the extra exports of
 * MKL/py/ssa_wrapper.c:47-123 (ssa_mkl_*). Prototypes, argument meaning, return codes and the
 * names of the struct fields that callers read are the reference's; the implementation runs on
 * an NVIDIA B200 (sm_100a): every call launches CUDA kernels on a stream owned by the context,
 * waits for them and mirrors the results (sigma, eigenvalues, U, V) into host arrays, so the
 * fields below are host memory exactly as in the reference.
 *
 * Differences a caller can observe (all documented, none changes a signature):
 *   - fft_len is next_pow2(N) (at least 32) instead of next_pow2(N + K - 1); circular
 *     correlation and convolution of length >= N never wrap for these lengths.
 *   - N is limited to 131072 per series; (k + oversampling) is limited to SSA_MAX_KP = 64.
 *     Larger requests return -1.
 *   - The Gaussian test matrix of ssa_opt_decompose_randomized comes from the library's own
 *     counter-based generator (seed 42, advancing per call) instead of MKL's MT2203 stream.
 *     ssa_opt_decompose_randomized_ex (ssa_b200.h) takes a caller-supplied matrix instead.
 *   - FFT convolutions and block products run in FP32; Gram accumulation, Cholesky,
 *     Rayleigh-Ritz eigen-solve and LRF/forecast run in FP64.
 *   - ssa_real is always double on this interface (the reference's SSA_USE_FLOAT build is not
 *     provided; the device computes in FP32 regardless).
 */
#ifndef SSA_OPT_R2C_H
#define SSA_OPT_R2C_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double ssa_real;

#define SSA_MAX_KP_API 64

struct ssa_gpu_ctx; /* device state: stream, device buffers, cached spectra */

/* Context of one series (reference: MKL/ssa_opt.h:145-225). Caller-allocated, zeroed by
 * ssa_opt_init, released by ssa_opt_free. sizeof(SSA_Opt) < 1024 (the ctypes buffer of
 * MKL/py/ssa_wrapper.py:92-94). */
typedef struct
{
    int N;
    int L;
    int K;
    int fft_len;
    int r2c_len;
    int batch_size;

    ssa_real *fft_x;      /* host copy of the signal spectrum, 2 * r2c_len doubles */
    ssa_real *ws_real;    /* host staging buffer (length max(N, fft_len)) */
    ssa_real *ws_complex; /* host staging buffer (2 * r2c_len) */
    ssa_real *ws_batch_real;    /* unused (NULL) */
    ssa_real *ws_batch_complex; /* unused (NULL) */

    ssa_real *U;           /* L x n_components, column-major (host) */
    ssa_real *V;           /* K x n_components, column-major (host) */
    ssa_real *sigma;       /* n_components, descending (host) */
    ssa_real *eigenvalues; /* sigma^2 (host) */
    int n_components;

    ssa_real *inv_diag_count; /* 1 / min(t+1, L, K, N-t), N values (host) */
    ssa_real *U_fft;          /* unused (NULL): cached spectra live on the device */
    ssa_real *V_fft;          /* unused (NULL) */
    bool fft_cached;          /* true after ssa_opt_cache_ffts */

    int prepared_kp;
    int prepared_lwork;       /* 0: no LAPACK workspace */
    ssa_real *decomp_Omega;   /* host buffer K x prepared_kp for a caller-supplied test matrix */
    ssa_real *decomp_Y;       /* unused (NULL) */
    bool prepared;

    bool initialized;
    bool decomposed;

    ssa_real total_variance;  /* sum of the computed eigenvalues */

    struct ssa_gpu_ctx *gpu;  /* device state (opaque) */
    uint64_t rng_calls;       /* test matrices drawn so far (generator stream position) */
} SSA_Opt;

/* reference: MKL/ssa_opt.h:228-248 */
typedef struct
{
    int n;
    ssa_real *singular_values;
    ssa_real *log_sv;
    ssa_real *gaps;
    ssa_real *cumulative_var;
    ssa_real *second_diff;
    int suggested_signal;
    ssa_real gap_threshold;
} SSA_ComponentStats;

/* reference: MKL/ssa_opt.h:251-268 */
typedef struct
{
    ssa_real *R;
    int L;
    ssa_real verticality;
    bool valid;
} SSA_LRF;

struct mssa_gpu_ctx;

/* reference: MKL/ssa_opt.h:271-315 */
typedef struct
{
    int M;
    int N;
    int L;
    int K;
    int fft_len;
    int r2c_len;
    ssa_real *U;           /* (M L) x n_components (host) */
    ssa_real *V;           /* K x n_components (host) */
    ssa_real *sigma;
    ssa_real *eigenvalues;
    int n_components;
    ssa_real *inv_diag_count;
    bool initialized;
    bool decomposed;
    ssa_real total_variance;
    struct mssa_gpu_ctx *gpu;
    uint64_t rng_calls;
} MSSA_Opt;

/* reference: MKL/ssa_opt.h:374-379 */
typedef struct
{
    int iterations;
    ssa_real final_diff;
    ssa_real converged;
} SSA_CadzowResult;

/* reference: MKL/ssa_opt.h:389-396 */
typedef struct
{
    ssa_real *periods;
    ssa_real *frequencies;
    ssa_real *moduli;
    ssa_real *rates;
    int n_components;
} SSA_ParEstimate;

/* reference: MKL/ssa_opt.h:407-413 */
typedef struct
{
    int iterations;
    ssa_real final_diff;
    int converged;
    int n_gaps;
} SSA_GapFillResult;

/* ---- core (reference MKL/ssa_opt.h:318-336) ---------------------------------------------- */
int ssa_opt_init(SSA_Opt *ssa, const ssa_real *x, int N, int L);
void ssa_opt_free(SSA_Opt *ssa);
int ssa_opt_decompose(SSA_Opt *ssa, int k, int max_iter);
int ssa_opt_decompose_block(SSA_Opt *ssa, int k, int block_size, int max_iter);
int ssa_opt_decompose_randomized(SSA_Opt *ssa, int k, int oversampling);
int ssa_opt_prepare(SSA_Opt *ssa, int max_k, int oversampling);
void ssa_opt_free_prepared(SSA_Opt *ssa);
int ssa_opt_update_signal(SSA_Opt *ssa, const ssa_real *new_x);
int ssa_opt_extend(SSA_Opt *ssa, int additional_k, int max_iter);
int ssa_opt_reconstruct(const SSA_Opt *ssa, const int *group, int n_group, ssa_real *output);
int ssa_opt_cache_ffts(SSA_Opt *ssa);
void ssa_opt_free_cached_ffts(SSA_Opt *ssa);

/* The Hankel matvec y = H v (v: K values, y: L values) and its adjoint z = H^T u (u: L values,
 * z: K values) on host arrays, computed on the device (reference MKL/ssa_opt.h:871-903, where
 * they are static functions that the reference's C tests call directly,
 * MKL/test/ssa_opt_test.c:1484, 1533). Nothing is written on an invalid context. The device
 * factor buffers serve as the workspace, so a decomposition the context holds is discarded
 * (decomposed becomes false). */
void ssa_opt_hankel_matvec(SSA_Opt *ssa, const ssa_real *v, ssa_real *y);
void ssa_opt_hankel_matvec_T(SSA_Opt *ssa, const ssa_real *u, ssa_real *z);

/* ---- analysis (reference MKL/ssa_opt.h:338-348) ------------------------------------------ */
int ssa_opt_wcorr_matrix(const SSA_Opt *ssa, ssa_real *W);
int ssa_opt_wcorr_matrix_fast(const SSA_Opt *ssa, ssa_real *W);
ssa_real ssa_opt_wcorr_pair(const SSA_Opt *ssa, int i, int j);
int ssa_opt_component_stats(const SSA_Opt *ssa, SSA_ComponentStats *stats);
void ssa_opt_component_stats_free(SSA_ComponentStats *stats);
int ssa_opt_find_periodic_pairs(const SSA_Opt *ssa, int *pairs, int max_pairs, ssa_real sv_tol, ssa_real wcorr_thresh);
int ssa_opt_compute_lrf(const SSA_Opt *ssa, const int *group, int n_group, SSA_LRF *lrf);
void ssa_opt_lrf_free(SSA_LRF *lrf);
int ssa_opt_forecast(const SSA_Opt *ssa, const int *group, int n_group, int n_forecast, ssa_real *output);
int ssa_opt_forecast_full(const SSA_Opt *ssa, const int *group, int n_group, int n_forecast, ssa_real *output);
int ssa_opt_forecast_with_lrf(const SSA_LRF *lrf, const ssa_real *base_signal, int base_len, int n_forecast, ssa_real *output);

/* ---- V-forecast (reference :352-355, MKL/ssa_opt.h:2906-3084): the per-step projection on the
 * group eigenvectors, evaluated as its equal LRF recurrence on the device (FP64); _fast starts
 * from the last L-1 values of base_signal ------------------------------------------------------ */
int ssa_opt_vforecast(const SSA_Opt *ssa, const int *group, int n_group, int n_forecast, ssa_real *output);
int ssa_opt_vforecast_full(const SSA_Opt *ssa, const int *group, int n_group, int n_forecast, ssa_real *output);
int ssa_opt_vforecast_fast(const SSA_Opt *ssa, const int *group, int n_group,
                           const ssa_real *base_signal, int base_len, int n_forecast, ssa_real *output);

/* ---- MSSA (reference :357-363) ------------------------------------------------------------ */
int mssa_opt_init(MSSA_Opt *mssa, const ssa_real *X, int M, int N, int L);
int mssa_opt_decompose(MSSA_Opt *mssa, int k, int oversampling);
int mssa_opt_reconstruct(const MSSA_Opt *mssa, int series_idx, const int *group, int n_group, ssa_real *output);
int mssa_opt_reconstruct_all(const MSSA_Opt *mssa, const int *group, int n_group, ssa_real *output);
int mssa_opt_series_contributions(const MSSA_Opt *mssa, ssa_real *contributions);
ssa_real mssa_opt_variance_explained(const MSSA_Opt *mssa, int start, int end);
void mssa_opt_free(MSSA_Opt *mssa);

/* ---- getters (reference :364-371) --------------------------------------------------------- */
int ssa_opt_get_trend(const SSA_Opt *ssa, ssa_real *output);
int ssa_opt_get_noise(const SSA_Opt *ssa, int noise_start, ssa_real *output);
ssa_real ssa_opt_variance_explained(const SSA_Opt *ssa, int start, int end);
int ssa_opt_get_singular_values(const SSA_Opt *ssa, ssa_real *output, int max_n);
int ssa_opt_get_eigenvalues(const SSA_Opt *ssa, ssa_real *output, int max_n);
ssa_real ssa_opt_get_total_variance(const SSA_Opt *ssa);

/* ---- Cadzow (reference :381-385) ---------------------------------------------------------- */
int ssa_opt_cadzow(const ssa_real *x, int N, int L, int rank, int max_iter, ssa_real tol,
                   ssa_real *output, SSA_CadzowResult *result);
int ssa_opt_cadzow_weighted(const ssa_real *x, int N, int L, int rank, int max_iter,
                            ssa_real tol, ssa_real alpha, ssa_real *output, SSA_CadzowResult *result);
int ssa_opt_cadzow_inplace(SSA_Opt *ssa, int rank, int max_iter, ssa_real tol, SSA_CadzowResult *result);

/* ---- ESPRIT and gap filling (reference :402-430): ESPRIT's cross Grams on the device, its
 * k x k solve and eigenvalues on the host; gap filling device-resident like Cadzow ----------- */
int ssa_opt_parestimate(const SSA_Opt *ssa, const int *group, int n_group, SSA_ParEstimate *result);
void ssa_opt_parestimate_free(SSA_ParEstimate *result);
int ssa_opt_gapfill(ssa_real *x, int N, int L, int rank, int max_iter, ssa_real tol, SSA_GapFillResult *result);
int ssa_opt_gapfill_simple(ssa_real *x, int N, int L, int rank, SSA_GapFillResult *result);

/* ---- shared-library extras (reference MKL/py/ssa_wrapper.c:47-123): CPU thread tuning of
 * MKL has no GPU counterpart; these keep the symbols and report a single "thread". --------- */
int ssa_mkl_init(int verbose);
int ssa_mkl_init_14900kf(int verbose);
int ssa_mkl_init_generic(int verbose);
void ssa_mkl_set_threads(int n);
int ssa_mkl_get_threads(void);
void ssa_mkl_get_cpu_info(int *p_cores, int *e_cores, int *is_hybrid, int *has_avx512);
void ssa_mkl_disable_affinity(void);

#ifdef __cplusplus
}
#endif

#include "ssa_b200.h"

#endif /* SSA_OPT_R2C_H */
