/*
 * MSSA (MKL/ssa_opt.h:3880-4283) and Cadzow (MKL/ssa_opt.h:3147-3442) entry points.
 * Placeholders that keep the exported symbols while the device implementation is built:
 * each returns the reference's failure value.
 */
#include <string.h>

#include "../../include/ssa_opt.h"

int mssa_opt_init(MSSA_Opt *mssa, const ssa_real *X, int M, int N, int L)
{
    if (mssa)
        memset(mssa, 0, sizeof(*mssa));
    (void)X, (void)M, (void)N, (void)L;
    return -1;
}
int mssa_opt_decompose(MSSA_Opt *mssa, int k, int oversampling)
{
    (void)mssa, (void)k, (void)oversampling;
    return -1;
}
int mssa_opt_decompose_ex(MSSA_Opt *mssa, int k, int oversampling, int power_iters, const double *Omega)
{
    (void)mssa, (void)k, (void)oversampling, (void)power_iters, (void)Omega;
    return -1;
}
int mssa_opt_reconstruct(const MSSA_Opt *mssa, int series_idx, const int *group, int n_group, ssa_real *output)
{
    (void)mssa, (void)series_idx, (void)group, (void)n_group, (void)output;
    return -1;
}
int mssa_opt_reconstruct_all(const MSSA_Opt *mssa, const int *group, int n_group, ssa_real *output)
{
    (void)mssa, (void)group, (void)n_group, (void)output;
    return -1;
}
int mssa_opt_series_contributions(const MSSA_Opt *mssa, ssa_real *contributions)
{
    (void)mssa, (void)contributions;
    return -1;
}
ssa_real mssa_opt_variance_explained(const MSSA_Opt *mssa, int start, int end)
{
    (void)mssa, (void)start, (void)end;
    return 0.0;
}
void mssa_opt_free(MSSA_Opt *mssa)
{
    if (mssa)
        memset(mssa, 0, sizeof(*mssa));
}

int ssa_opt_cadzow(const ssa_real *x, int N, int L, int rank, int max_iter, ssa_real tol, ssa_real *output,
                   SSA_CadzowResult *result)
{
    (void)x, (void)N, (void)L, (void)rank, (void)max_iter, (void)tol, (void)output, (void)result;
    return -1;
}
int ssa_opt_cadzow_weighted(const ssa_real *x, int N, int L, int rank, int max_iter, ssa_real tol, ssa_real alpha,
                            ssa_real *output, SSA_CadzowResult *result)
{
    (void)x, (void)N, (void)L, (void)rank, (void)max_iter, (void)tol, (void)alpha, (void)output, (void)result;
    return -1;
}
int ssa_opt_cadzow_inplace(SSA_Opt *ssa, int rank, int max_iter, ssa_real tol, SSA_CadzowResult *result)
{
    (void)ssa, (void)rank, (void)max_iter, (void)tol, (void)result;
    return -1;
}
