/*
 * Internal extensions of the uneven-batch pipeline (ssa_ragged.c) used by the request server
 * (ssa_server.c): per-series generator seeds, capture of the forecast group's LRF into
 * caller-owned device memory, and access to the packed device outputs.
 */
#ifndef SSA_RAGGED_INT_H
#define SSA_RAGGED_INT_H

#include <cuda_runtime_api.h>
#include <stddef.h>

#include "../../include/ssa_opt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Group slot (index into the batch's groups) whose reconstruction the LRF uses, and the component
 * indices that define the LRF (copied to the device). */
int ssar_set_lrf_group(ssa_rbatch *rb, int slot, const int *group, int n_group);
/* Enqueue a run on device input d_x (packed). seeds[s] (or NULL) is the generator seed of series
 * s; lrf_dst[s] (or NULL, or a NULL entry) receives R (L-1), tail (L-1) and verticality (1)
 * doubles of the forecast group; series whose k does not cover the group are skipped. */
int ssar_run_enqueue_ex(ssa_rbatch *rb, int B, const int *N, const int *L, const int *k, const double *d_x,
                        const unsigned long long *seeds, double *const *lrf_dst, const unsigned char *want_w);
/* Follow-up run on resident factors, no decomposition: series s has k[s] components with
 * factors U[s] (L x k, leading dimension round4(L)), V[s] (K x k, round4(K)), FP32, and sigma[s]
 * (k doubles), all in device memory, and its own group gidx[goff[s] .. goff[s+1]) (host). The run
 * writes the group's reconstruction (N doubles at the series' groups offset, group slot 0) and,
 * where lrf_dst[s] is non-NULL, the group's R (L-1), reconstruction tail (L-1) and verticality.
 * Indices >= k[s] are skipped. The batch must have been created with at least one group. */
int ssar_run_followup(ssa_rbatch *rb, int B, const int *N, const int *L, const int *k, const float *const *U,
                      const float *const *V, const double *const *sig, const int *gidx, const int *goff,
                      double *const *lrf_dst);
/* Device factor blocks of series s of the last decomposition run (U: L x k', leading dimension
 * round4(L); V: K x k', round4(K)); returns k' or -1. Valid until the next run. */
int ssar_series_factors(const ssa_rbatch *rb, int s, const float **U, const float **V);
/* Cadzow iterations (the device-resident loop of ssa_opt_cadzow) on the host signal x. With y1
 * (host, N values) given, it is taken as the first rank-`rank` projection of x: the first
 * iteration measures it against x instead of decomposing, and the loop continues from it.
 * Returns the iteration count or -1 (ssa_api.c). */
int ssab_cadzow_from(const double *x, const double *y1, int N, int L, int rank, int max_iter, double tol,
                     double *output, SSA_CadzowResult *result);
cudaStream_t ssar_main_stream(const ssa_rbatch *rb);
/* FFT-length bucket a series of length N runs in (0 .. SSAR_NB - 1), and a bucket's stream after
 * a run (NULL for a bucket the run did not use). Outside graph replays, work a caller enqueues
 * on a bucket's stream after ssar_run_enqueue_ex follows that bucket's part of the run and
 * nothing else. */
#define SSAR_NB 20
int ssar_bucket_index(int N);
cudaStream_t ssar_bucket_stream(const ssa_rbatch *rb, int g);
const int *ssar_status(const ssa_rbatch *rb);
const int *ssar_lrf_status(const ssa_rbatch *rb);
const double *ssar_sigma(const ssa_rbatch *rb);
const double *ssar_W(const ssa_rbatch *rb);
const double *ssar_groups(const ssa_rbatch *rb);
const size_t *ssar_offsets(const ssa_rbatch *rb);
void ssar_totals(const ssa_rbatch *rb, size_t *t4);
size_t ssar_series_bytes(int N, int L, int k, int p, int n_groups);
/* The library's stream-ordered device memory pool (current device), blocks cached on free. */
cudaMemPool_t ssar_pool(void);

#ifdef __cplusplus
}
#endif
#endif
