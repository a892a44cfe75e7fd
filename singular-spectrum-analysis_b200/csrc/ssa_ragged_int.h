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
cudaStream_t ssar_main_stream(const ssa_rbatch *rb);
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
