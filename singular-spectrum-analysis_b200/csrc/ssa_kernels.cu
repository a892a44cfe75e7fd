// sm_100a kernels for the SSA decomposition / reconstruction hot path.
//
// Kernel map (reference call sites in SSA-Opt MKL/ssa_opt.h):
//   k_spectrum     FFT(x ‖ 0) of the signal (:1255-1257) and cached component spectra
//                  FFT(sigma_i u_i), FFT(v_i) (:2110-2245)
//   k_corr         Hankel matvec block Y = H V / adjoint Z = H^T U (:910-1004): R2C of each
//                  column, product with conj of the column spectrum, C2R, first L (or K) values;
//                  with a NULL input the column is the device Gaussian test matrix (:1719)
//   k_gram         FP64-accumulated Gram partials A^T W A (CholQR2 Gram, Rayleigh-Ritz Gram and
//                  the W-correlation SYRK :2543 with diagonal-count weights)
//   k_chol         FP64 Cholesky of the (k+p) x (k+p) Gram and its triangular inverse
//   k_rowmul       C = A * Bsmall row by row (Q = Y R^{-1}, U = Q Z, V = B Z Sigma^{-1}; :1736)
//   k_rr           FP64 Jacobi eigen-decomposition of B^T B: sigma, Ritz rotations, sign rule
//                  sum U[:, i] >= 0 (:1741-1759)
//   k_elem_recon   fused elementary reconstruction x~_i = inv_w * (sigma_i u_i conv v_i) and its
//                  weighted norm (reconstruct :2325-2400 for one component, no cached spectra)
//   k_recon        grouped reconstruction from cached spectra (:2338-2356, :2393-2397)
//   k_wfin         W = G_ij / sqrt(G_ii G_jj) (:2527-2546)
//   k_lrf          LRF coefficients with the verticality check and the R-forecast recurrence
//                  (:2766-2841), FP64
#include "ssa_fft.cuh"
#include "ssa_kernels.h"

#include <atomic>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

using namespace ssa;

static std::atomic<unsigned long long> g_launches{0};

// Device-side self-check record: {violations, kernel id, block, code, value}. Kernels that
// validate their job write the first violation here and skip the work of that block.
__device__ unsigned int g_ssa_check[5];

__device__ __forceinline__ void check_fail(unsigned kernel, unsigned code, unsigned value) {
    if (atomicAdd(&g_ssa_check[0], 1u) == 0) {
        g_ssa_check[1] = kernel;
        g_ssa_check[2] = blockIdx.x + 65536u * blockIdx.y;
        g_ssa_check[3] = code;
        g_ssa_check[4] = value;
    }
}

extern "C" int ssad_read_checks(unsigned int* out5, int reset) {
    cudaError_t e = cudaMemcpyFromSymbol(out5, g_ssa_check, sizeof(unsigned int) * 5);
    if (e != cudaSuccess) return (int)e;
    if (reset) {
        unsigned int z[5] = {0, 0, 0, 0, 0};
        e = cudaMemcpyToSymbol(g_ssa_check, z, sizeof(z));
    }
    return (int)e;
}
static inline int launched(cudaError_t e) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return (int)e;
}

extern "C" unsigned long long ssad_launch_count(void) { return g_launches.load(); }
// Kernels launched by a CUDA-graph replay (the launches the graph captured).
extern "C" void ssad_count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ---------------------------------------------------------------------------------------------
// Device-side helpers
// ---------------------------------------------------------------------------------------------

// SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014).
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Two N(0,1) values for rows (2*pair, 2*pair+1) of generated column `col` (Box-Muller on two
// 24-bit uniforms taken from one 64-bit hash of (seed, col, pair)).
__device__ __forceinline__ float2 gauss_pair(unsigned long long seed, int col, int pair) {
    unsigned long long key = mix64(seed ^ (0xD1B54A32D192ED03ull * (unsigned long long)(col + 1)));
    unsigned long long z = mix64(key + (unsigned long long)pair);
    float u1 = ((float)(z >> 40) + 1.0f) * (1.0f / 16777216.0f);        // (0, 1]
    float u2 = (float)((z >> 16) & 0xFFFFFFull) * (1.0f / 16777216.0f);  // [0, 1)
    float r = sqrtf(-2.0f * logf(u1));
    float sn, cs;
    sincospif(2.0f * u2, &sn, &cs);
    return make_float2(r * cs, r * sn);
}

__device__ __forceinline__ int diag_count(int t, int N, int L, int K) {
    int c = min(min(t + 1, L), min(K, N - t));
    return c > 0 ? c : 1;
}

__device__ __forceinline__ bool edge_diag(int t, int N) { return t < SSA_EDGE || t >= N - SSA_EDGE; }

// sum_{i + j = t} u[i] v[j] over 0 <= i < L, 0 <= j < K, in FP64 (at most SSA_EDGE terms on an
// edge anti-diagonal).
__device__ __forceinline__ double diag_sum(const float* __restrict__ u, const float* __restrict__ v, int t, int L,
                                           int K) {
    const int i0 = max(0, t - K + 1), i1 = min(t, L - 1);
    double s = 0.0;
    for (int i = i0; i <= i1; ++i) s = fma((double)u[i], (double)v[t - i], s);
    return s;
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* red) {
    // red: >= 32 entries of shared scratch; returns the total to every thread. Fixed order.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (warp == 0) {
        T t = lane < nw ? red[lane] : T(0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) red[0] = t;
    }
    __syncthreads();
    T r = red[0];
    __syncthreads();
    return r;
}

__host__ __device__ __forceinline__ int pk_index(int i, int j, int n) {  // i <= j
    return i * n - (i * (i - 1)) / 2 + (j - i);
}

// Load column `c` of job J into the packed buffer s (input, generated, or double signal).
// Packed input point z[i] = (a[2i], a[2i+1]) of one column (zero from n on), read from global
// memory by the first FFT pass: FP32 (times sc), FP64, or generated N(0,1) pairs.
struct ColPts {
    const float* f32;
    const double* f64;
    float sc;
    int n;
    unsigned long long seed;
    int col;
    static constexpr bool kSmem = false;
    // packed points that can be nonzero
    __device__ __forceinline__ int nz() const { return (n + 1) >> 1; }
    __device__ __forceinline__ float2 operator()(int i) const {
        const int t = 2 * i;
        float2 v = make_float2(0.f, 0.f);
        if (t < n) {
            if (f32) {
                // columns start 8-byte aligned and t is even: one 8-byte load for the pair
                if (t + 1 < n) {
                    v = *reinterpret_cast<const float2*>(f32 + t);
                    v.x *= sc;
                    v.y *= sc;
                } else {
                    v.x = f32[t] * sc;
                }
            } else if (f64) {
                v.x = (float)f64[t];
                v.y = t + 1 < n ? (float)f64[t + 1] : 0.f;
            } else {
                v = gauss_pair(seed, col, i);
                if (t + 1 >= n) v.y = 0.f;
            }
        }
        return v;
    }
};

// Input column c of a job: its FP32 column (scaled by scale[c]), else its FP64 column, else the
// generated Gaussian test column col0 + c.
__device__ __forceinline__ ColPts col_pts(const ssa_col_job& J, int c) {
    ColPts p;
    p.f32 = J.in ? J.in + (long long)c * J.ld_in : nullptr;
    p.f64 = (!J.in && J.in64) ? J.in64 + (long long)c * J.ld_in : nullptr;
    p.sc = (J.in && J.scale) ? (float)J.scale[c] : 1.0f;
    p.n = J.n_in;
    p.seed = J.seedp ? *J.seedp : J.seed;
    p.col = J.col0 + c;
    return p;
}

// Output point Z[i] written by the last FFT pass as the reals out[2i], out[2i+1] (times sc),
// the first n reals only.
struct RealOut {
    float* out;
    int n;
    float sc;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void operator()(int i, float2 v) const {
        const int t = 2 * i;
        if (t + 1 < n)
            *reinterpret_cast<float2*>(out + t) = make_float2(v.x * sc, v.y * sc);
        else if (t < n)
            out[t] = v.x * sc;
    }
};

template <int LOGH>
__device__ __forceinline__ void load_column(float2* s, const ssa_col_job& J, int c) {
    constexpr int H = 1 << LOGH;
    if (J.in) {
        const float sc = J.scale ? (float)J.scale[c] : 1.0f;
        load_real<LOGH>(s, J.in + (long long)c * J.ld_in, J.n_in, sc);
    } else if (J.in64) {
        const double* a = J.in64 + (long long)c * J.ld_in;
        const int n = J.n_in;
        for (int i = threadIdx.x; i < H; i += blockDim.x) {
            const int r = 2 * i;
            float2 v;
            v.x = r < n ? (float)a[r] : 0.f;
            v.y = r + 1 < n ? (float)a[r + 1] : 0.f;
            s[spad(i)] = v;
        }
    } else {
        const int n = J.n_in;
        const int col = J.col0 + c;
        const unsigned long long seed = J.seedp ? *J.seedp : J.seed;
        for (int i = threadIdx.x; i < H; i += blockDim.x) {
            const int r = 2 * i;
            float2 v = make_float2(0.f, 0.f);
            if (r < n) {
                v = gauss_pair(seed, col, i);
                if (r + 1 >= n) v.y = 0.f;
            }
            s[spad(i)] = v;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// FFT column kernels
// ---------------------------------------------------------------------------------------------

template <int LOGH>
__global__ void __launch_bounds__(FftShape<LOGH>::BLOCK, FftShape<LOGH>::MINB) k_spectrum(const ssa_col_job* __restrict__ jobs) {
    constexpr int H = 1 << LOGH;
    extern __shared__ float2 smem[];
    const ssa_col_job J = jobs[blockIdx.y];
    const int c = blockIdx.x;
    if (c >= J.ncols) return;
    float2* tw = smem + spad_size(H);
    load_twiddles<LOGH + 1>(tw);
    fft_block_io<LOGH, false>(smem, col_pts(J, c), SmemPts{smem}, tw);
    float2* out = reinterpret_cast<float2*>(J.spec + (long long)c * J.ld_spec);
    for (int k = threadIdx.x; k <= H / 2; k += blockDim.x) {
        if (k == 0) {
            float2 z0 = smem[spad(0)];
            out[0] = make_float2(z0.x + z0.y, 0.f);
            out[H] = make_float2(z0.x - z0.y, 0.f);
        } else {
            float2 ak, am;
            unpack_pair<LOGH>(smem[spad(k)], smem[spad(H - k)], wm<LOGH>(tw, k), ak, am);
            out[k] = ak;
            out[H - k] = am;
        }
    }
}

// Spectral product stage of a correlation sweep on the packed transform Z of one column held in
// s (H points, NT threads, thread tid): unpack the real spectrum A, form P = X conj(A) with the
// signal spectrum X (H + 1 bins, A[0] and A[H] real) and pack P for the inverse transform, in
// place. Thread tid takes the bin pairs (k, H - k), k = tid + i NT; the spectrum bins of GMAX
// such pairs are read (read-only path) before any of them is used, so that their L2 latency
// overlaps. Bin H/2, its own mirror, goes to thread 0 last.
template <int LOGH, int NT, int GMAX>
__device__ __forceinline__ void corr_product(float2* s, const float2* __restrict__ X, const float2* tw, int tid) {
    constexpr int H = 1 << LOGH;
    constexpr int NI = (H / 2 + NT - 1) / NT;
    constexpr int G = NI < GMAX ? NI : GMAX;
#pragma unroll 1
    for (int i0 = 0; i0 < NI; i0 += G) {
        float2 xk[G], xm[G];
#pragma unroll
        for (int i = 0; i < G; ++i) {
            const int k = tid + (i0 + i) * NT;
            if (i0 + i < NI && k < H / 2) {
                xk[i] = __ldg(X + k);
                xm[i] = __ldg(X + (H - k));  // k = 0: the Nyquist bin X[H]
            }
        }
#pragma unroll
        for (int i = 0; i < G; ++i) {
            const int k = tid + (i0 + i) * NT;
            if (i0 + i >= NI || k >= H / 2) continue;
            float2 zk, zm;
            if (k == 0) {
                const float2 z0 = s[spad(0)];
                pack_pair(cscale(xk[i], z0.x + z0.y), cscale(xm[i], z0.x - z0.y), make_float2(1.f, 0.f), zk, zm);
                s[spad(0)] = zk;
            } else {
                const float2 w = wm<LOGH>(tw, k);
                float2 ak, am;
                unpack_pair<LOGH>(s[spad(k)], s[spad(H - k)], w, ak, am);
                pack_pair(cmulc(xk[i], ak), cmulc(xm[i], am), w, zk, zm);
                s[spad(k)] = zk;
                s[spad(H - k)] = zm;
            }
        }
    }
    if (tid == 0) {
        constexpr int k = H / 2;
        const float2 x = __ldg(X + k), w = wm<LOGH>(tw, k), z = s[spad(k)];
        float2 ak, am, zk, zm;
        unpack_pair<LOGH>(z, z, w, ak, am);
        pack_pair(cmulc(x, ak), cmulc(x, am), w, zk, zm);
        s[spad(k)] = zm;  // the pair's mirror slot is the same slot
    }
}

// Work unit of a correlation sweep: the grid (columns, jobs), one CTA per column; or, with a
// column list of ntiles (job, column) tiles, one CTA (cluster) per tile, so that no CTA is spent
// on the columns beyond a job's ncols. Returns the unit's (job, column), or false past the end.
__device__ __forceinline__ bool sweep_column(const ssa_tile* __restrict__ tiles, int ntiles, int unit, int& job,
                                             int& c) {
    if (tiles) {
        if (unit >= ntiles) return false;
        const ssa_tile t = tiles[unit];
        job = t.job;
        c = t.c0;
    } else {
        job = blockIdx.y;
        c = unit;
    }
    return true;
}

// (A persistent form of this kernel, resident CTAs looping over the column list, measured 0.9%
// faster on real length 32768 but made the one-pass form of the (columns, jobs) grid 20% slower
// on the uniform batches: not kept.)
template <int LOGH>
__global__ void __launch_bounds__(FftShape<LOGH>::BLOCK, FftShape<LOGH>::MINB) k_corr(const ssa_col_job* __restrict__ jobs,
                                                                                       const ssa_tile* __restrict__ tiles,
                                                                                       int ntiles) {
    constexpr int H = 1 << LOGH;
    extern __shared__ float2 smem[];
    int jb, c;
    if (!sweep_column(tiles, ntiles, blockIdx.x, jb, c)) return;
    const ssa_col_job J = jobs[jb];
    if (c >= J.ncols) return;
    float2* tw = smem + spad_size(H);
    load_twiddles<LOGH + 1>(tw);
    fft_block_io<LOGH, false>(smem, col_pts(J, c), SmemPts{smem}, tw);
    corr_product<LOGH, FftShape<LOGH>::BLOCK, 4>(smem, reinterpret_cast<const float2*>(J.X), tw, threadIdx.x);
    __syncthreads();
    fft_block_io<LOGH, true>(smem, SmemPts{smem}, RealOut{J.out + (long long)c * J.ld_out, J.n_out, 1.0f / (float)H},
                             tw);
}

// The correlation of k_corr from the input column's real spectrum A (H + 1 bins: A[0], A[H] real,
// as k_spectrum writes it): P = conj-product with the signal spectrum, packed and transformed
// back. Bit-identical to k_corr on the same column (the spectrum holds the same FP32 values k_corr
// forms in registers).
template <int LOGH>
__global__ void __launch_bounds__(FftShape<LOGH>::BLOCK, FftShape<LOGH>::MINB) k_corr_spec(const ssa_col_job* __restrict__ jobs) {
    constexpr int H = 1 << LOGH;
    extern __shared__ float2 smem[];
    const ssa_col_job J = jobs[blockIdx.y];
    const int c = blockIdx.x;
    if (c >= J.ncols) return;
    float2* tw = smem + spad_size(H);
    load_twiddles<LOGH + 1>(tw);
    __syncthreads();
    const float2* X = reinterpret_cast<const float2*>(J.X);
    const float2* A = reinterpret_cast<const float2*>(J.spec + (long long)c * J.ld_spec);
    for (int k = threadIdx.x; k <= H / 2; k += blockDim.x) {
        float2 zk, zm;
        if (k == 0) {
            if (X) pack_pair(cscale(__ldg(X), A[0].x), cscale(__ldg(X + H), A[H].x), make_float2(1.f, 0.f), zk, zm);
            else pack_pair(A[0], A[H], make_float2(1.f, 0.f), zk, zm);
            smem[spad(0)] = zk;
        } else {
            const float2 w = wm<LOGH>(tw, k);
            if (X) pack_pair(cmulc(__ldg(X + k), A[k]), cmulc(__ldg(X + (H - k)), A[H - k]), w, zk, zm);
            else pack_pair(A[k], A[H - k], w, zk, zm);
            smem[spad(k)] = zk;
            smem[spad(H - k)] = zm;
        }
    }
    __syncthreads();
    fft_block_io<LOGH, true>(smem, SmemPts{smem}, RealOut{J.out + (long long)c * J.ld_out, J.n_out, 1.0f / (float)H},
                             tw);
}

// One channel's term of a stacked adjoint sweep: the forward transform of input column c and its
// conj-product with the channel's signal spectrum, written (first channel) or added into the
// column's product accumulator (spec + c ld_spec, H + 1 bins). The channels of one accumulator
// run as consecutive launches on one stream.
template <int LOGH>
__global__ void __launch_bounds__(FftShape<LOGH>::BLOCK, FftShape<LOGH>::MINB) k_corr_acc(const ssa_col_job* __restrict__ jobs,
                                                                                           int first) {
    constexpr int H = 1 << LOGH;
    extern __shared__ float2 smem[];
    const ssa_col_job J = jobs[blockIdx.y];
    const int c = blockIdx.x;
    if (c >= J.ncols) return;
    float2* tw = smem + spad_size(H);
    load_twiddles<LOGH + 1>(tw);
    fft_block_io<LOGH, false>(smem, col_pts(J, c), SmemPts{smem}, tw);
    const float2* X = reinterpret_cast<const float2*>(J.X);
    float2* acc = reinterpret_cast<float2*>(J.spec + (long long)c * J.ld_spec);
    for (int k = threadIdx.x; k <= H / 2; k += blockDim.x) {
        float2 pk, pm;
        if (k == 0) {
            const float2 z0 = smem[spad(0)];
            pk = cscale(__ldg(X), z0.x + z0.y);
            pm = cscale(__ldg(X + H), z0.x - z0.y);
        } else {
            float2 ak, am;
            unpack_pair<LOGH>(smem[spad(k)], smem[spad(H - k)], wm<LOGH>(tw, k), ak, am);
            pk = cmulc(__ldg(X + k), ak);
            pm = cmulc(__ldg(X + (H - k)), am);
        }
        const int km = k == 0 ? H : H - k;  // k = H / 2 is its own mirror: pk == pm there
        if (!first) {
            pk = cadd(pk, acc[k]);
            pm = cadd(pm, acc[km]);
        }
        acc[k] = pk;
        acc[km] = pm;
    }
}

// ---------------------------------------------------------------------------------------------
// Multi-length persistent correlation sweep
// ---------------------------------------------------------------------------------------------

// Points a tile's unused column slots read: none (n = 0), so they load nothing from global memory.
__device__ __forceinline__ ColPts idle_pts() {
    ColPts p;
    p.f32 = nullptr;
    p.f64 = nullptr;
    p.sc = 0.f;
    p.n = 0;
    p.seed = 0;
    p.col = 0;
    return p;
}

// Shared-memory floats2 of the multi-length kernel: the largest data region over the lengths
// (2^(13 - logh) padded buffers of H points, largest at the smallest length) plus the twiddle
// table of the largest length.
__host__ __device__ constexpr int multi_data_f2() {
    return (1 << (SSA_MULTI_MAX_LOGH - SSA_MULTI_MIN_LOGH)) * spad_size(1 << SSA_MULTI_MIN_LOGH);
}
__host__ __device__ constexpr int multi_smem_f2() { return multi_data_f2() + TwSplit<SSA_MULTI_MAX_LOGH + 1>::N; }

// One tile at length H = 2^LOGH: column slot g of the CTA (threads g T .. g T + T - 1, T = H / 16)
// runs column c0 + g of the job as k_corr does, in its own padded buffer.
template <int LOGH>
__device__ __forceinline__ void corr_tile(float2* smem, const ssa_col_job* __restrict__ Jp, int c0) {
    const ssa_col_job& J = *Jp;  // fields read where used (no copy held across the transform)
    constexpr int H = 1 << LOGH;
    constexpr int T = H / 16;
    static_assert(512 % T == 0, "whole column slots per CTA");
    const int g = threadIdx.x / T, tid = threadIdx.x - g * T;
    const int c = c0 + g;
    const bool valid = c < J.ncols;
    float2* s = smem + g * spad_size(H);
    float2* tw = smem + multi_data_f2();
    load_twiddles<LOGH + 1>(tw);  // published by the first pass's closing barrier
    const SmemPts sp{s};
    fft_passes<LOGH, false, 0>(s, valid ? col_pts(J, c) : idle_pts(), sp, tw, tid);
    if (valid) corr_product<LOGH, T, 4>(s, reinterpret_cast<const float2*>(J.X), tw, tid);
    __syncthreads();
    const RealOut ro{valid ? J.out + (long long)c * J.ld_out : nullptr, valid ? J.n_out : 0, 1.0f / (float)H};
    fft_passes<LOGH, true, 0>(s, sp, ro, tw, tid);
}

__global__ void __launch_bounds__(512, 2) k_corr_multi(const ssa_col_job* __restrict__ jobs,
                                                        const ssa_tile* __restrict__ tiles, int ntiles,
                                                        int* __restrict__ head) {
    extern __shared__ float2 smem[];
    __shared__ int s_tile;
    for (;;) {
        __syncthreads();  // the previous tile is done with the buffers, the table and s_tile
        if (threadIdx.x == 0) s_tile = atomicAdd(head, 1);
        __syncthreads();
        const int t = s_tile;
        if (t >= ntiles) return;
        const ssa_tile T = tiles[t];
        const ssa_col_job* J = jobs + T.job;
        switch (T.logh) {
            case 8: corr_tile<8>(smem, J, T.c0); break;
            case 9: corr_tile<9>(smem, J, T.c0); break;
            case 10: corr_tile<10>(smem, J, T.c0); break;
            case 11: corr_tile<11>(smem, J, T.c0); break;
            case 12: corr_tile<12>(smem, J, T.c0); break;
            case 13: corr_tile<13>(smem, J, T.c0); break;
            default: check_fail(20, 1, (unsigned)T.logh); break;
        }
    }
}

// Elementary reconstruction of component c: x~[t] = inv_w[t] * (sigma_c u_c conv v_c)[t], and
// norm2[c] = sum_t w[t] x~[t]^2 (w = diagonal count).
template <int LOGH>
__global__ void __launch_bounds__(FftShape<LOGH>::BLOCK) k_elem_recon(const ssa_col_job* __restrict__ jobs) {
    constexpr int H = 1 << LOGH;
    extern __shared__ float2 smem[];
    __shared__ double red[32];
    float2* s1 = smem;
    float2* s2 = smem + spad_size(H);
    float2* tw = smem + 2 * spad_size(H);
    const ssa_col_job J = jobs[blockIdx.y];
    const int c = blockIdx.x;
    if (c >= J.ncols) return;
    const float sc = J.scale ? (float)J.scale[c] : 1.0f;
    load_twiddles<LOGH + 1>(tw);
    fft_block_io<LOGH, false>(s1, ColPts{J.in + (long long)c * J.ld_in, nullptr, sc, J.n_in, 0, 0}, SmemPts{s1}, tw);
    fft_block_io<LOGH, false>(s2, ColPts{J.in2 + (long long)c * J.ld_in2, nullptr, 1.0f, J.n_in2, 0, 0}, SmemPts{s2},
                              tw);
    for (int k = threadIdx.x; k <= H / 2; k += blockDim.x) {
        float2 zk, zm;
        if (k == 0) {
            const float2 a0 = s1[spad(0)], b0 = s2[spad(0)];
            const float p0 = (a0.x + a0.y) * (b0.x + b0.y);
            const float ph = (a0.x - a0.y) * (b0.x - b0.y);
            pack_pair(make_float2(p0, 0.f), make_float2(ph, 0.f), make_float2(1.f, 0.f), zk, zm);
            s1[spad(0)] = zk;
        } else {
            const float2 w = wm<LOGH>(tw, k);
            float2 ak, am, bk, bm;
            unpack_pair<LOGH>(s1[spad(k)], s1[spad(H - k)], w, ak, am);
            unpack_pair<LOGH>(s2[spad(k)], s2[spad(H - k)], w, bk, bm);
            pack_pair(cmul(ak, bk), cmul(am, bm), w, zk, zm);
            s1[spad(k)] = zk;
            s1[spad(H - k)] = zm;
        }
    }
    __syncthreads();
    fft_block<LOGH, true>(s1, tw);
    float* out = J.out + (long long)c * J.ld_out;
    const float inv_h = 1.0f / (float)H;
    const float* u = J.in + (long long)c * J.ld_in;
    const float* vv = J.in2 + (long long)c * J.ld_in2;
    double acc = 0.0;
    for (int t = threadIdx.x; t < J.N; t += blockDim.x) {
        const float2 z = s1[spad(t >> 1)];
        double p = (double)(((t & 1) ? z.y : z.x) * inv_h);
        if (edge_diag(t, J.N)) p = (double)sc * diag_sum(u, vv, t, J.n_in, J.n_in2);
        const int cnt = diag_count(t, J.N, J.L, J.K);
        out[t] = (float)(p / (double)cnt);
        acc += p * p / (double)cnt;
    }
    acc = block_sum<double>(acc, red);
    if (threadIdx.x == 0 && J.norm2) J.norm2[c] = acc;
}

// Elementary reconstruction with one FFT buffer: the spectrum of sigma_c u_c (bins 0..H of the
// real length-2H transform, as k_spectrum writes it) comes from global memory; v_c is transformed
// in shared memory. Same outputs as k_elem_recon.
template <int LOGH>
__global__ void __launch_bounds__(FftShape<LOGH>::BLOCK) k_elem_recon1(const ssa_col_job* __restrict__ jobs) {
    constexpr int H = 1 << LOGH;
    extern __shared__ float2 smem[];
    __shared__ double red[32];
    float2* s2 = smem;
    float2* tw = smem + spad_size(H);
    const ssa_col_job J = jobs[blockIdx.y];
    const int c = blockIdx.x;
    if (c >= J.ncols) return;
    load_twiddles<LOGH + 1>(tw);
    fft_block_io<LOGH, false>(s2, ColPts{J.in2 + (long long)c * J.ld_in2, nullptr, 1.0f, J.n_in2, 0, 0}, SmemPts{s2},
                              tw);
    const float2* us = reinterpret_cast<const float2*>(J.spec + (long long)c * J.ld_spec);
    for (int k = threadIdx.x; k <= H / 2; k += blockDim.x) {
        float2 zk, zm;
        if (k == 0) {
            const float2 b0 = s2[spad(0)];
            const float p0 = us[0].x * (b0.x + b0.y);
            const float ph = us[H].x * (b0.x - b0.y);
            pack_pair(make_float2(p0, 0.f), make_float2(ph, 0.f), make_float2(1.f, 0.f), zk, zm);
            s2[spad(0)] = zk;
        } else {
            const float2 w = wm<LOGH>(tw, k);
            float2 bk, bm;
            unpack_pair<LOGH>(s2[spad(k)], s2[spad(H - k)], w, bk, bm);
            pack_pair(cmul(us[k], bk), cmul(us[H - k], bm), w, zk, zm);
            s2[spad(k)] = zk;
            s2[spad(H - k)] = zm;
        }
    }
    __syncthreads();
    fft_block<LOGH, true>(s2, tw);
    float* out = J.out + (long long)c * J.ld_out;
    const float inv_h = 1.0f / (float)H;
    const float sc = J.scale ? (float)J.scale[c] : 1.0f;
    const float* u = J.in + (long long)c * J.ld_in;
    const float* vv = J.in2 + (long long)c * J.ld_in2;
    double acc = 0.0;
    for (int t = threadIdx.x; t < J.N; t += blockDim.x) {
        const float2 z = s2[spad(t >> 1)];
        double p = (double)(((t & 1) ? z.y : z.x) * inv_h);
        if (edge_diag(t, J.N)) p = (double)sc * diag_sum(u, vv, t, J.n_in, J.n_in2);
        const int cnt = diag_count(t, J.N, J.L, J.K);
        out[t] = (float)(p / (double)cnt);
        acc += p * p / (double)cnt;
    }
    acc = block_sum<double>(acc, red);
    if (threadIdx.x == 0 && J.norm2) J.norm2[c] = acc;
}

// Group sums of an uneven batch: one job per series.
__global__ void k_group_sum_ragged(const ssa_rgsum_job* __restrict__ jobs, const int* __restrict__ group_idx,
                                   const int* __restrict__ group_off) {
    const ssa_rgsum_job J = jobs[blockIdx.z];
    const int g = blockIdx.y;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= J.N) return;
    const int* gi = J.gidx ? J.gidx : group_idx + group_off[g];
    const int gn = J.gidx ? J.gn : group_off[g + 1] - group_off[g];
    if (J.gidx && g > 0) return;  // a job's own group is its only one
    double acc = 0.0;
    for (int e = 0; e < gn; ++e) {
        const int i = gi[e];
        if (i < 0 || i >= J.k) continue;
        acc += (double)J.recon[(long long)i * J.ld_recon + t];
    }
    J.out[(long long)g * J.N + t] = acc;
}

// Grouped reconstruction from cached spectra.
template <int LOGH>
__global__ void __launch_bounds__(FftShape<LOGH>::BLOCK, FftShape<LOGH>::MINB) k_recon(const ssa_recon_job* __restrict__ jobs) {
    constexpr int H = 1 << LOGH;
    extern __shared__ float2 smem[];
    const ssa_recon_job J = jobs[blockIdx.y];
    float2* tw = smem + spad_size(H);
    load_twiddles<LOGH + 1>(tw);
    __syncthreads();
    for (int k = threadIdx.x; k <= H / 2; k += blockDim.x) {
        float2 pk = make_float2(0.f, 0.f), pm = make_float2(0.f, 0.f);
        for (int g = 0; g < J.n_group; ++g) {
            const int i = J.group[g];
            if (i < 0 || i >= J.k) continue;
            const float2* us = reinterpret_cast<const float2*>(J.Us + (long long)i * J.ld_spec);
            const float2* vs = reinterpret_cast<const float2*>(J.Vs + (long long)i * J.ld_spec);
            const float2 a = cmul(us[k], vs[k]);
            const float2 b = cmul(us[H - k], vs[H - k]);
            pk = cadd(pk, a);
            pm = cadd(pm, b);
        }
        float2 zk, zm;
        if (k == 0) {
            pack_pair(pk, pm, make_float2(1.f, 0.f), zk, zm);
            smem[spad(0)] = zk;
        } else {
            pack_pair(pk, pm, wm<LOGH>(tw, k), zk, zm);
            smem[spad(k)] = zk;
            smem[spad(H - k)] = zm;
        }
    }
    __syncthreads();
    fft_block<LOGH, true>(smem, tw);
    const float inv_h = 1.0f / (float)H;
    for (int t = threadIdx.x; t < J.N; t += blockDim.x) {
        const float2 z = smem[spad(t >> 1)];
        double p = (double)(((t & 1) ? z.y : z.x) * inv_h);
        if (J.U && edge_diag(t, J.N)) {
            p = 0.0;
            for (int g = 0; g < J.n_group; ++g) {
                const int i = J.group[g];
                if (i < 0 || i >= J.k) continue;
                p += (double)(float)J.sigma[i] *
                     diag_sum(J.U + (long long)i * J.ldU, J.V + (long long)i * J.ldV, t, J.L, J.K);
            }
        }
        const double v = p / (double)diag_count(t, J.N, J.L, J.K);
        if (J.out64) J.out64[t] = v;
        if (J.out) J.out[t] = (float)v;
    }
}

// ---------------------------------------------------------------------------------------------
// Gram partials (FP64 accumulation of FP32 data)
// ---------------------------------------------------------------------------------------------

#define GRAM_THREADS 128
#define GSTR (SSA_GRAM_CHUNK + 1)
// Column stride of the staged chunk ([col][row] floats): 132 = 4 (mod 32), so the fragment
// loads of a warp (row 4s + t, column 8b + g for lane 4g + t) hit 32 distinct banks, and a
// column starts 16-byte aligned for the 16-byte asynchronous copies.
#define GRAM_S (SSA_GRAM_CHUNK + 4)
#define GRAM_STAGE (SSA_MAX_KP * GRAM_S)
#define GRAM_SMEM (2 * GRAM_STAGE * (int)sizeof(float))

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, int bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// D = A B + D for one 8x8 FP64 tile (FP64 tensor cores; lane 4g + t holds A[g][t], B[t][g],
// D[g][2t], D[g][2t + 1]).
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

#define GRAM_MMA_THREADS 256
#define GRAM_HALF (SSA_GRAM_CHUNK / 2)

// Stage rows [r0 + 64 h, r0 + 64 h + 64) of columns [0, n) into rows [64 h, 64 h + 64) of buf
// ([col][row], stride GRAM_S), by the 128 threads of half h; rows at or beyond r_end are
// zero-filled (they belong to another CTA's partial or lie past m).
__device__ __forceinline__ void gram_stage_half(uint32_t buf, const ssa_gram_job& J, int r0, int r_end, bool vec,
                                                int h, int th) {
    const int rb = r0 + GRAM_HALF * h;
    const uint32_t hb = buf + 4u * (uint32_t)(GRAM_HALF * h);
    if (vec) {
        constexpr int Q = GRAM_HALF / 4;
        for (int idx = th; idx < J.n * Q; idx += GRAM_MMA_THREADS / 2) {
            const int col = idx / Q, q = idx - col * Q;
            const int r = rb + 4 * q;
            const int valid = min(4, max(0, r_end - r));
            const float* src = valid > 0 ? J.A + (long long)r + (long long)col * J.ld : J.A;
            cp_async16(hb + 4u * (uint32_t)(col * GRAM_S + 4 * q), src, 4 * valid);
        }
    } else {
        for (int idx = th; idx < J.n * GRAM_HALF; idx += GRAM_MMA_THREADS / 2) {
            const int col = idx / GRAM_HALF, q = idx - col * GRAM_HALF;
            const int r = rb + q;
            const bool ok = r < r_end;
            const float* src = ok ? J.A + (long long)r + (long long)col * J.ld : J.A;
            cp_async4(hb + 4u * (uint32_t)(col * GRAM_S + q), src, ok ? 4 : 0);
        }
    }
}

// Named barrier of one half of the CTA (ids 1 and 2 as immediates, so that only three of the
// CTA's barriers are in use).
__device__ __forceinline__ void bar_half(int h) {
    if (h) asm volatile("bar.sync 2, %0;" ::"n"(GRAM_MMA_THREADS / 2) : "memory");
    else asm volatile("bar.sync 1, %0;" ::"n"(GRAM_MMA_THREADS / 2) : "memory");
}

// The chunk loop of warp pair (WQ, WQ + 4): tile columns c1 = WQ (rows 0 .. WQ, when
// 2 WQ <= nt - 1) and c2 = nt - 1 - WQ (rows 0 .. c2, when c2 > WQ), accumulator slot i <= WQ
// for (i, c1) and WQ + 1 + i for (i, c2). With WQ a compile-time constant every slot and every
// row fragment has a fixed register, so each fragment of A is loaded and converted once per
// k-step for both tile columns (8 - WQ fragments instead of 9 loads).
template <bool WEIGHTED, int WQ>
__device__ __forceinline__ void gram_loop(const ssa_gram_job& J, const float* gsm, uint32_t sbase, int r_begin,
                                          int r_end, int nchunk, bool vec, int nt, int half, int th, int lane,
                                          double (&acc)[9][2], double& csum) {
    const int g = lane >> 2, t = lane & 3;
    const bool has1 = 2 * WQ <= nt - 1;
    const int c2 = (has1 && nt - 1 - WQ > WQ) ? nt - 1 - WQ : -1;
    for (int ic = 0; ic < nchunk; ++ic) {
        const int r0 = r_begin + ic * SSA_GRAM_CHUNK;
        if (ic + 1 < nchunk)
            gram_stage_half(sbase + 4u * (uint32_t)(((ic + 1) & 1) * GRAM_STAGE), J, r0 + SSA_GRAM_CHUNK, r_end, vec,
                            half, th);
        cp_async_commit();
        cp_async_wait<1>();
        bar_half(half);
        const float* sA = gsm + (ic & 1) * GRAM_STAGE;
        if (J.colsum && th < J.n) {
            double cs = 0.0;
            for (int r = 0; r < GRAM_HALF; ++r) cs += (double)sA[th * GRAM_S + GRAM_HALF * half + r];
            csum += cs;
        }
        if (has1) {
            const float* pa = sA + g * GRAM_S + t;  // lane's element of tile row 0, k-step 0
#pragma unroll 2
            for (int s4 = half * GRAM_HALF; s4 < (half + 1) * GRAM_HALF; s4 += 4) {
                const float* row = pa + s4;
                double w = 1.0;
                if (WEIGHTED) w = (double)diag_count(r0 + s4 + t, J.N, J.L, J.K);
                const double b1 = w * (double)row[8 * WQ * GRAM_S];
                const double b2 = c2 >= 0 ? w * (double)row[8 * c2 * GRAM_S] : 0.0;
#pragma unroll
                for (int bi = 0; bi < 8; ++bi) {
                    if (bi > WQ && bi > c2) break;
                    const double a = (double)row[8 * bi * GRAM_S];
                    if (bi <= WQ) dmma_8x8x4(acc[bi][0], acc[bi][1], a, b1);
                    if (bi <= 7 - WQ && bi <= c2) dmma_8x8x4(acc[WQ + 1 + bi][0], acc[WQ + 1 + bi][1], a, b2);
                }
            }
        }
        bar_half(half);  // this half of the stage is refilled two chunks later
    }
}

// Gram partials on the FP64 tensor cores: part[chunk] = A_c^T W A_c over this CTA's rows, FP32
// data, exact FP64 products (FP32 x FP32 x integer weight), FP64 accumulation. G is cut into
// 8x8 tiles (nt = ceil(n/8) <= 8 per side); warps w and w + 4 own the upper-triangle tiles of
// tile columns w and nt - 1 - w (at most nt + 1 <= 9 tiles), warp w over the first half of each
// chunk's rows and warp w + 4 over the second half (their sums are added at the end). Each half
// of the CTA stages its own half of every chunk (asynchronous copies into two buffers, the next
// chunk landing while the current one is multiplied) and synchronises on its own named barrier,
// so the two halves do not wait for each other between chunks.
template <bool WEIGHTED>
__global__ void __launch_bounds__(GRAM_MMA_THREADS, 3) k_gram(const ssa_gram_job* __restrict__ jobs) {
    extern __shared__ __align__(16) float gsm[];
    const ssa_gram_job J = jobs[blockIdx.y];
    const int chunk = blockIdx.x;
    const int r_begin = chunk * J.rows_per_cta;
    if (r_begin >= J.m) return;
    const int r_end = min(J.m, r_begin + J.rows_per_cta);
    const int n = J.n;
    const int nt = (n + 7) >> 3;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wq = warp & 3, half = warp >> 2;
    const int th = threadIdx.x & (GRAM_MMA_THREADS / 2 - 1);
    const int g = lane >> 2, t = lane & 3;
    const int c1 = 2 * wq <= nt - 1 ? wq : -1;
    const int c2 = (c1 >= 0 && nt - 1 - wq > wq) ? nt - 1 - wq : -1;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(gsm);
    const bool vec = ((reinterpret_cast<uintptr_t>(J.A) & 15) == 0) && ((J.ld & 3) == 0);
    // padding columns n .. 8 nt - 1 of both stages read as zeros
    for (int idx = threadIdx.x; idx < (8 * nt - n) * SSA_GRAM_CHUNK; idx += GRAM_MMA_THREADS) {
        const int col = n + idx / SSA_GRAM_CHUNK, q = idx % SSA_GRAM_CHUNK;
        gsm[col * GRAM_S + q] = 0.f;
        gsm[GRAM_STAGE + col * GRAM_S + q] = 0.f;
    }
    __syncthreads();
    double acc[9][2];
#pragma unroll
    for (int i = 0; i < 9; ++i) acc[i][0] = acc[i][1] = 0.0;
    double csum = 0.0;
    const int nchunk = (r_end - r_begin + SSA_GRAM_CHUNK - 1) / SSA_GRAM_CHUNK;
    gram_stage_half(sbase, J, r_begin, r_end, vec, half, th);
    cp_async_commit();
    switch (wq) {
        case 0: gram_loop<WEIGHTED, 0>(J, gsm, sbase, r_begin, r_end, nchunk, vec, nt, half, th, lane, acc, csum); break;
        case 1: gram_loop<WEIGHTED, 1>(J, gsm, sbase, r_begin, r_end, nchunk, vec, nt, half, th, lane, acc, csum); break;
        case 2: gram_loop<WEIGHTED, 2>(J, gsm, sbase, r_begin, r_end, nchunk, vec, nt, half, th, lane, acc, csum); break;
        default: gram_loop<WEIGHTED, 3>(J, gsm, sbase, r_begin, r_end, nchunk, vec, nt, half, th, lane, acc, csum); break;
    }
    // the second row half's sums join the first half's through shared memory, once both halves
    // are done with the stages
    __syncthreads();
    double* red = reinterpret_cast<double*>(gsm);
    if (half == 1 && c1 >= 0) {
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            red[((wq * 9 + i) * 2 + 0) * 32 + lane] = acc[i][0];
            red[((wq * 9 + i) * 2 + 1) * 32 + lane] = acc[i][1];
        }
    }
    double* csred = red + 4 * 9 * 2 * 32;
    if (half == 1 && J.colsum && th < n) csred[th] = csum;
    __syncthreads();
    double* part = J.part + (long long)chunk * (n * (n + 1) / 2);
    if (half == 0 && c1 >= 0) {
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            acc[i][0] += red[((wq * 9 + i) * 2 + 0) * 32 + lane];
            acc[i][1] += red[((wq * 9 + i) * 2 + 1) * 32 + lane];
        }
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const bool first = i <= c1;
            const int bi = first ? i : i - c1 - 1;
            if (!first && (c2 < 0 || bi > c2)) continue;
            const int row = 8 * bi + g;
            const int cb = 8 * (first ? c1 : c2) + 2 * t;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int col = cb + h;
                if (row < n && col < n && row <= col) part[pk_index(row, col, n)] = acc[i][h];
            }
        }
    }
    if (half == 0 && J.colsum && th < n) J.colsum[(long long)chunk * n + th] = csum + csred[th];
}

// ---------------------------------------------------------------------------------------------
// Cholesky + triangular inverse (FP64, one CTA per job)
// ---------------------------------------------------------------------------------------------

#define SMALL_THREADS 256
#define SLD (SSA_MAX_KP + 1)
#define SMALL_SMEM (2 * SSA_MAX_KP * SLD * (int)sizeof(double))

// Sum the packed-upper Gram partials into the symmetric column-major matrix G (ld SLD). Each
// thread owns up to four packed entries and walks the chunks four at a time, so that sixteen
// independent loads of the (L2-resident) partials are in flight: the sum over chunks is a
// latency chain otherwise, and it sets the latency of the small per-series kernels.
__device__ void reduce_packed(const double* __restrict__ part, int nchunks, int n, double* G) {
    const int np = n * (n + 1) / 2;
    const int bs = blockDim.x;
    for (int e0 = threadIdx.x; e0 < np; e0 += 4 * bs) {
        int e[4];
        double acc[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            e[u] = e0 + u * bs;
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
        }
        int c = 0;
        for (; c + 4 <= nchunks; c += 4) {
#pragma unroll
            for (int v = 0; v < 4; ++v)
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (e[u] < np) acc[u][v] += part[(long long)(c + v) * np + e[u]];
        }
        for (; c < nchunks; ++c)
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (e[u] < np) acc[u][0] += part[(long long)c * np + e[u]];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (e[u] >= np) continue;
            // packed row-major upper triangle: row i starts at i n - i (i - 1) / 2
            int i = 0;
            while (i + 1 < n && (i + 1) * n - ((i + 1) * i) / 2 <= e[u]) ++i;
            const int j = i + (e[u] - (i * n - (i * (i - 1)) / 2));
            const double sum = (acc[u][0] + acc[u][1]) + (acc[u][2] + acc[u][3]);
            G[j * SLD + i] = sum;
            G[i * SLD + j] = sum;
        }
    }
}

// Largest diagonal entry (>= 0) of G, or -1 when a diagonal entry is not finite.
__device__ double diag_max(const double* G, int n, double* red) {
    double dm = 0.0;
    int bad = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double d = G[i * SLD + i];
        if (!isfinite(d)) bad = 1;
        dm = fmax(dm, d);
    }
    for (int o = 16; o > 0; o >>= 1) {
        dm = fmax(dm, __shfl_down_sync(0xffffffffu, dm, o));
        bad |= __shfl_down_sync(0xffffffffu, bad, o);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = bad ? -1.0 : dm;
    __syncthreads();
    double m = 0.0;
    int b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        if (red[w] < 0.0) b = 1;
        m = fmax(m, red[w]);
    }
    __syncthreads();
    return b ? -1.0 : m;
}

// In-place Cholesky G = R^T R of the symmetric column-major G (ld SLD): on return G holds R
// (upper, R[r][c] at G[c * SLD + r]) with zeros below the diagonal. Pivots below `floor_` are
// raised to it: directions that small are rounding noise of a rank-deficient input.
__device__ void chol_upper_inplace(double* G, int n, double floor_) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int j = 0; j < n; ++j) {
        // every thread reads the pivot before anyone overwrites it
        double d = G[j * SLD + j];
        if (!(d > floor_)) d = floor_;
        d = sqrt(d);
        const double inv = 1.0 / d;
        __syncthreads();
        if (threadIdx.x == 0) G[j * SLD + j] = d;
        for (int c = j + 1 + threadIdx.x; c < n; c += blockDim.x) G[c * SLD + j] *= inv;
        __syncthreads();
        // trailing update of the upper triangle: rows r > j (one warp per row), columns c >= r
        for (int r = j + 1 + warp; r < n; r += nw) {
            const double rjr = G[r * SLD + j];
            for (int c = r + lane; c < n; c += 32) G[c * SLD + r] -= rjr * G[c * SLD + j];
        }
        __syncthreads();
    }
    for (int c = warp; c < n; c += nw)
        for (int r = c + 1 + lane; r < n; r += 32) G[c * SLD + r] = 0.0;
    __syncthreads();
}

// X = R^{-1} for the upper-triangular R in G (both column-major, ld SLD), by row sweeps from the
// bottom: X[i][j] = (delta_ij - sum_{l=i+1..j} R[i][l] X[l][j]) / R[i][i]. Four threads per
// column split each sum (blockDim.x = SMALL_THREADS = 256 covers n <= 64 columns).
__device__ void tri_inv_upper(const double* G, double* X, int n) {
    const int j = threadIdx.x >> 2, q = threadIdx.x & 3;
    for (int i = n - 1; i >= 0; --i) {
        double s = 0.0;
        if (j < n && j > i)
            for (int l = i + 1 + q; l <= j; l += 4) s = fma(G[l * SLD + i], X[j * SLD + l], s);
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        if (j < n && q == 0) X[j * SLD + i] = j >= i ? ((j == i ? 1.0 : 0.0) - s) / G[i * SLD + i] : 0.0;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(SMALL_THREADS) k_chol(const ssa_chol_job* __restrict__ jobs) {
    extern __shared__ double dsm[];
    __shared__ double red[32];
    double* G = dsm;
    const ssa_chol_job J = jobs[blockIdx.x];
    const int n = J.n;
    reduce_packed(J.part, J.nchunks, n, G);
    __syncthreads();
    const double dmax = diag_max(G, n, red);
    if (dmax < 0.0) {
        if (threadIdx.x == 0 && J.status) atomicOr(J.status, 1);
    }
    const double floor_ = dmax > 0.0 ? dmax * 1e-13 * (double)n : 1.0;
    chol_upper_inplace(G, n, floor_);
    double* X = dsm + SSA_MAX_KP * SLD;
    tri_inv_upper(G, X, n);
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int c = e / n, r = e - c * n;
        J.Rinv[e] = X[c * SLD + r];
    }
}

// ---------------------------------------------------------------------------------------------
// Row products with a small matrix: C = A Bm (or sub - A Bm), FP32 register tiles
// ---------------------------------------------------------------------------------------------

#define RM_THREADS 256
#define RM_ROWS SSA_ROWMUL_ROWS
// A block [col][row] (column stride 132: 16-byte aligned columns), Bm [k][j] (row stride 68:
// 16-byte aligned rows; the staging stores, k fastest across lanes, meet 8 banks).
#define RM_SA (RM_ROWS + 4)
#define RM_SB (SSA_MAX_KP + 4)
#define RM_SMEM (SSA_MAX_KP * RM_SA * (int)sizeof(float) + SSA_MAX_KP * RM_SB * (int)sizeof(float) + \
                 (RM_THREADS / 32) * SSA_MAX_KP * (int)sizeof(double))

// One CTA per SSA_ROWMUL_ROWS rows: the rows of A (all n columns) land in shared memory by
// asynchronous copies while Bm (FP32, or FP64 rounded to FP32) is staged beside them. Warp w
// owns output columns [8 w, 8 w + 8) and lane l rows [4 l, 4 l + 4): per k one 16-byte load of
// A (4 rows), two broadcast 16-byte loads of Bm (8 columns) and 32 FMAs. For an upper-triangular
// Bm (R^{-1} of a CholQR pass) warp w stops at k = 8 w + 7, past which its columns are zero.
__global__ void __launch_bounds__(RM_THREADS) k_rowmul(const ssa_rowmul_job* __restrict__ jobs) {
    extern __shared__ __align__(16) unsigned char rsm[];
    float* sA = reinterpret_cast<float*>(rsm);
    float* sB = sA + SSA_MAX_KP * RM_SA;
    double* wsum = reinterpret_cast<double*>(sB + SSA_MAX_KP * RM_SB);
    const ssa_rowmul_job J = jobs[blockIdx.y];
    const int n = J.n, p = J.p;
    const int r0 = blockIdx.x * RM_ROWS;
    if (r0 >= J.m) return;
    const int rows = min(RM_ROWS, J.m - r0);
    const uint32_t abase = (uint32_t)__cvta_generic_to_shared(sA);
    const bool vec = ((reinterpret_cast<uintptr_t>(J.A) & 15) == 0) && ((J.lda & 3) == 0);
    if (vec) {
        constexpr int Q = RM_ROWS / 4;
        for (int idx = threadIdx.x; idx < n * Q; idx += RM_THREADS) {
            const int col = idx / Q, r = 4 * (idx - col * Q);
            const int valid = min(4, max(0, rows - r));
            const float* src = valid > 0 ? J.A + (long long)(r0 + r) + (long long)col * J.lda : J.A;
            cp_async16(abase + 4u * (uint32_t)(col * RM_SA + r), src, 4 * valid);
        }
    } else {
        for (int idx = threadIdx.x; idx < n * RM_ROWS; idx += RM_THREADS) {
            const int col = idx / RM_ROWS, r = idx - col * RM_ROWS;
            const bool ok = r < rows;
            const float* src = ok ? J.A + (long long)(r0 + r) + (long long)col * J.lda : J.A;
            cp_async4(abase + 4u * (uint32_t)(col * RM_SA + r), src, ok ? 4 : 0);
        }
    }
    cp_async_commit();
    {
        // Bm column-major: k fastest across lanes (coalesced), all loads of a thread in flight
        // together before the stores
        constexpr int IT = SSA_MAX_KP * SSA_MAX_KP / RM_THREADS;
        float bv[IT];
#pragma unroll
        for (int u = 0; u < IT; ++u) {
            const int idx = threadIdx.x + u * RM_THREADS;
            const int k = idx & (SSA_MAX_KP - 1), j = idx / SSA_MAX_KP;
            float v = 0.f;
            if (k < n && j < p)
                v = J.Bm64 ? (float)J.Bm64[k + (long long)j * J.ldb] : J.Bm[k + (long long)j * J.ldb];
            bv[u] = v;
        }
#pragma unroll
        for (int u = 0; u < IT; ++u) {
            const int idx = threadIdx.x + u * RM_THREADS;
            sB[(idx & (SSA_MAX_KP - 1)) * RM_SB + idx / SSA_MAX_KP] = bv[u];
        }
    }
    cp_async_wait<0>();
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c0 = 8 * warp;  // this warp's columns
    const int rl = 4 * lane;  // this lane's rows
    float acc[4][8];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = 0.f;
    if (c0 < p) {
        const int kend = J.Bm64 ? min(n, c0 + 8) : n;  // R^{-1} is upper triangular
#pragma unroll 4
        for (int k = 0; k < kend; ++k) {
            const float4 a = *reinterpret_cast<const float4*>(sA + k * RM_SA + rl);
            const float4 b0 = *reinterpret_cast<const float4*>(sB + k * RM_SB + c0);
            const float4 b1 = *reinterpret_cast<const float4*>(sB + k * RM_SB + c0 + 4);
            const float av[4] = {a.x, a.y, a.z, a.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 8; ++v) acc[u][v] = fmaf(av[u], bv[v], acc[u][v]);
        }
    }
    // a lane's four rows of a column are contiguous: one 16-byte store (and load of sub) per
    // column when C (and sub) allow it, so a warp writes 512 contiguous bytes
    const bool vecC = rl + 4 <= rows && ((reinterpret_cast<uintptr_t>(J.C) & 15) == 0) && ((J.ldc & 3) == 0) &&
                      (!J.sub || (((reinterpret_cast<uintptr_t>(J.sub) & 15) == 0) && ((J.ldsub & 3) == 0)));
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        const int col = c0 + v;
        double cs = 0.0;
        if (col < p) {
            float x[4] = {acc[0][v], acc[1][v], acc[2][v], acc[3][v]};
            const long long cb = (long long)(r0 + rl) + (long long)col * J.ldc;
            if (vecC) {
                if (J.sub) {
                    const float4 sv =
                        *reinterpret_cast<const float4*>(J.sub + (long long)(r0 + rl) + (long long)col * J.ldsub);
                    x[0] = sv.x - x[0];
                    x[1] = sv.y - x[1];
                    x[2] = sv.z - x[2];
                    x[3] = sv.w - x[3];
                }
                *reinterpret_cast<float4*>(J.C + cb) = make_float4(x[0], x[1], x[2], x[3]);
#pragma unroll
                for (int u = 0; u < 4; ++u) cs += (double)x[u];
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (rl + u < rows) {
                        if (J.sub) x[u] = J.sub[(long long)(r0 + rl + u) + (long long)col * J.ldsub] - x[u];
                        J.C[cb + u] = x[u];
                        cs += (double)x[u];
                    }
                }
            }
        }
        if (J.colsum) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) cs += __shfl_xor_sync(0xffffffffu, cs, o);
            if (lane == 0 && col < p) wsum[warp * SSA_MAX_KP + col] = cs;
        }
    }
    if (J.colsum) {
        __syncthreads();
        for (int j = threadIdx.x; j < p; j += RM_THREADS) J.colsum[(long long)blockIdx.x * p + j] = wsum[(j >> 3) * SSA_MAX_KP + j];
    }
}

// ---------------------------------------------------------------------------------------------
// Rayleigh-Ritz: FP64 parallel cyclic Jacobi on G_B = B^T B
// ---------------------------------------------------------------------------------------------

#define RR_THREADS 512

// Round-robin (circle method) position i after `step` rotations of positions 1 .. ne-1 (each
// rotation moves the last position's index to position 1): pairs (pos(t), pos(ne-1-t)) of one
// step are disjoint and every pair meets once per ne-1 steps.
__device__ __forceinline__ int rr_pos(int i, int step, int ne) {
    if (i == 0) return 0;
    const int m = ne - 1;
    int v = (i - 1 - step) % m;
    if (v < 0) v += m;
    return 1 + v;
}

// One-sided (Hestenes) Jacobi on the n columns of A (column c at A + c * SLD, FP64, shared
// memory): A <- A J with J a product of plane rotations accumulated into Z (initialised by the
// caller), until every column pair is orthogonal to 4 sqrt(n) eps relative (rotations below the
// rounding level of the dot products would otherwise never stop; LAPACK's one-sided Jacobi uses
// sqrt(m) eps). Round-robin pairing computed from the step number; one half-warp per pair (so
// the up to 32 pairs of a step run side by side in 16 warps), lanes own rows l, l + 16, l + 32,
// l + 48; one barrier per step. The rotation angle follows Rutishauser's formula written as
//   t = sign(zeta) |2 gamma| / (|beta - alpha| + sqrt((beta - alpha)^2 + 4 gamma^2)),
//   zeta = (beta - alpha) / (2 gamma),   c = 1 / sqrt(1 + t^2),   s = c t,
// which is the same t without the intermediate quotient. On return nrm[c] = ||A[:, c]||.
// Called by every thread of the block.
__device__ void onesided_jacobi(double* A, double* Z, int n, int* notconv, double* nrm) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int half = lane >> 4, l16 = lane & 15;
    const int ne = (n + 1) & ~1;  // even count; index n is a dummy when n is odd
    const int npairs = ne / 2;
    const double tiny = 1e-300;
    const double tol = 4.0 * sqrt((double)n) * 2.220446049250313e-16;
    const double tol2 = tol * tol;
    for (int sweep = 0; sweep < 40; ++sweep) {
        if (threadIdx.x == 0) *notconv = 0;
        __syncthreads();
        for (int step = 0; step < ne - 1; ++step) {
            // warp-uniform trip count: both halves of a warp run the same iterations
            for (int t0 = 2 * warp; t0 < npairs; t0 += 2 * nw) {
                const int t = t0 + half;
                int p = t < npairs ? rr_pos(t, step, ne) : n;
                int q = t < npairs ? rr_pos(ne - 1 - t, step, ne) : n;
                if (p < 0 || q < 0) {
                    if (l16 == 0) check_fail(6, 6, (unsigned)(p * 1000 + q));
                    p = q = n;
                }
                const bool live = p < n && q < n;
                double* ap = A + (live ? p : 0) * SLD;
                double* aq = A + (live ? q : 0) * SLD;
                double al = 0.0, be = 0.0, ga = 0.0;
                if (live) {
#pragma unroll
                    for (int i = 0; i < SSA_MAX_KP / 16; ++i) {
                        const int r = l16 + 16 * i;
                        if (r < n) {
                            const double x = ap[r], y = aq[r];
                            al = fma(x, x, al);
                            be = fma(y, y, be);
                            ga = fma(x, y, ga);
                        }
                    }
                }
#pragma unroll
                for (int o = 8; o > 0; o >>= 1) {
                    al += __shfl_xor_sync(0xffffffffu, al, o);
                    be += __shfl_xor_sync(0xffffffffu, be, o);
                    ga += __shfl_xor_sync(0xffffffffu, ga, o);
                }
                if (live && fabs(ga) > tiny && ga * ga > tol2 * (al * be)) {
                    if (l16 == 0) *notconv = 1;
                    const double d = be - al, g2 = 2.0 * ga;
                    const double mag = fabs(g2) / (fabs(d) + sqrt(fma(d, d, g2 * g2)));
                    const double tt = ((d >= 0.0) == (g2 >= 0.0) || d == 0.0) ? mag : -mag;
                    const double cs = rsqrt(fma(tt, tt, 1.0));
                    const double sn = cs * tt;
                    double* zp = Z + p * SLD;
                    double* zq = Z + q * SLD;
#pragma unroll
                    for (int i = 0; i < SSA_MAX_KP / 16; ++i) {
                        const int r = l16 + 16 * i;
                        if (r < n) {
                            const double x = ap[r], y = aq[r];
                            ap[r] = cs * x - sn * y;
                            aq[r] = sn * x + cs * y;
                            const double u = zp[r], v = zq[r];
                            zp[r] = cs * u - sn * v;
                            zq[r] = sn * u + cs * v;
                        }
                    }
                }
            }
            __syncthreads();
        }
        // Every thread reads the flag before thread 0 may reset it for the next sweep; otherwise
        // warps could leave the loop at different sweeps and desynchronise the barriers.
        const bool converged = !*notconv;
        __syncthreads();
        if (converged) break;
    }
    for (int c = warp; c < n; c += nw) {
        double s = 0.0;
        for (int r = lane; r < n; r += 32) s = fma(A[c * SLD + r], A[c * SLD + r], s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) nrm[c] = sqrt(s);
    }
    __syncthreads();
}

// Rayleigh-Ritz: B^T B = R^T R (FP64 Cholesky), then one-sided (Hestenes) Jacobi on the
// columns of R: R Z = W Sigma with orthonormal Z, so B^T B = Z Sigma^2 Z^T. One warp per column
// pair of a round-robin step; each lane owns rows lane and lane + 32.
__global__ void __launch_bounds__(RR_THREADS) k_rr(const ssa_rr_job* __restrict__ jobs) {
    extern __shared__ double dsm[];
    double* A = dsm;                    // column c at A + c * SLD
    double* Z = dsm + SSA_MAX_KP * SLD;
    __shared__ double qs[SSA_MAX_KP];
    __shared__ double nrm[SSA_MAX_KP];
    __shared__ int order[SSA_MAX_KP];
    __shared__ double red[32];
    __shared__ int notconv;
    const ssa_rr_job J = jobs[blockIdx.x];
    const int n = J.kp;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    {
        unsigned code = 0, val = 0;
        if (n < 1 || n > SSA_MAX_KP) code = 1, val = (unsigned)n;
        else if (J.k < 1 || J.k > n) code = 2, val = (unsigned)J.k;
        else if (J.nchunks < 1 || J.nchunks > (1 << 16)) code = 3, val = (unsigned)J.nchunks;
        else if (J.nchunks_q < 1 || J.nchunks_q > (1 << 16)) code = 4, val = (unsigned)J.nchunks_q;
        else if (!J.part || !J.qsum || !J.sigma || !J.Zu || !J.Zv || !J.status) code = 5;
        if (code) {
            if (threadIdx.x == 0) check_fail(6, code, val);
            return;
        }
    }
    reduce_packed(J.part, J.nchunks, n, A);
    for (int c = warp; c < n; c += nw)
        for (int r = lane; r < n; r += 32) Z[c * SLD + r] = (r == c) ? 1.0 : 0.0;
    for (int l = threadIdx.x; l < n; l += blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < J.nchunks_q; ++c) s += J.qsum[(long long)c * n + l];
        qs[l] = s;
    }
    __syncthreads();
    const double dmax = diag_max(A, n, red);
    if (dmax < 0.0) {
        if (threadIdx.x == 0 && J.status) atomicOr(J.status, 2);
    }
    chol_upper_inplace(A, n, dmax > 0.0 ? dmax * 1e-15 : 1.0);
    onesided_jacobi(A, Z, n, &notconv, nrm);
    __syncthreads();
    // descending singular values: each column's rank is the number of columns before it
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = nrm[i];
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const double w = nrm[j];
            rank += (w > v) || (w == v && j < i);
        }
        order[rank] = i;
    }
    __syncthreads();
    const int k = J.k;
    for (int j = warp; j < k; j += nw) {
        const int col = order[j];
        if (col < 0 || col >= n) {
            if (lane == 0) check_fail(6, 7, (unsigned)col);
            continue;
        }
        const double sg = nrm[col];
        double dot = 0.0;
        for (int l = lane; l < n; l += 32) dot = fma(qs[l], Z[col * SLD + l], dot);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
        const double sgn = dot < 0.0 ? -1.0 : 1.0;
        const double isg = sg > 1e-300 ? 1.0 / sg : 0.0;
        for (int l = lane; l < n; l += 32) {
            const double z = sgn * Z[col * SLD + l];
            J.Zu[l + j * n] = (float)z;
            J.Zv[l + j * n] = (float)(z * isg);
        }
        if (lane == 0) {
            J.sigma[j] = sg;
            if (!isfinite(sg) && J.status) atomicOr(J.status, 2);
        }
    }
}


// ---------------------------------------------------------------------------------------------
// Block power iteration support (reference MKL/ssa_opt.h:1765-1933): cross Grams for deflation
// and the block Rayleigh quotient, small SVD, final ordering
// ---------------------------------------------------------------------------------------------

#define XG_SMEM (2 * SSA_MAX_KP * GSTR * (int)sizeof(float))

__global__ void __launch_bounds__(GRAM_THREADS) k_xgram(const ssa_xgram_job* __restrict__ jobs) {
    extern __shared__ float xsm[];
    float* sA = xsm;
    float* sB = xsm + SSA_MAX_KP * GSTR;
    const ssa_xgram_job J = jobs[blockIdx.y];
    const int chunk = blockIdx.x;
    const int r_begin = chunk * J.rows_per_cta;
    if (r_begin >= J.m) return;
    const int r_end = min(J.m, r_begin + J.rows_per_cta);
    const int na = J.na, nb = J.nb;
    const int tba = (na + 3) >> 2, tbb = (nb + 3) >> 2;
    const int ntiles = tba * tbb;
    double acc[2][4][4];
    int ti[2], tj[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int t = threadIdx.x + q * GRAM_THREADS;
        ti[q] = t < ntiles ? t / tbb : -1;
        tj[q] = t < ntiles ? t - (t / tbb) * tbb : -1;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[q][a][b] = 0.0;
    }
    for (int r0 = r_begin; r0 < r_end; r0 += SSA_GRAM_CHUNK) {
        const int rows = min(SSA_GRAM_CHUNK, r_end - r0);
        __syncthreads();
        for (int idx = threadIdx.x; idx < SSA_MAX_KP * SSA_GRAM_CHUNK; idx += GRAM_THREADS) {
            const int col = idx / SSA_GRAM_CHUNK, r = idx - col * SSA_GRAM_CHUNK;
            float va = 0.f, vb = 0.f;
            if (r < rows) {
                if (col < na) va = J.A[(long long)(r0 + r) + (long long)col * J.lda];
                if (col < nb) vb = J.B[(long long)(r0 + r) + (long long)col * J.ldb];
            }
            sA[col * GSTR + r] = va;
            sB[col * GSTR + r] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (ti[q] < 0) continue;
            const float* pa = sA + (ti[q] * 4) * GSTR;
            const float* pb = sB + (tj[q] * 4) * GSTR;
            for (int r = 0; r < rows; ++r) {
                double x[4], y[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    x[u] = (double)pa[u * GSTR + r];
                    y[u] = (double)pb[u * GSTR + r];
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int v = 0; v < 4; ++v) acc[q][u][v] = fma(x[u], y[v], acc[q][u][v]);
            }
        }
    }
    double* part = J.part + (long long)chunk * na * nb;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        if (ti[q] < 0) continue;
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int i = ti[q] * 4 + u, j = tj[q] * 4 + v;
                if (i < na && j < nb) part[i * nb + j] = acc[q][u][v];
            }
    }
}

__global__ void k_xreduce(const ssa_xreduce_job* __restrict__ jobs) {
    const ssa_xreduce_job J = jobs[blockIdx.x];
    const int tot = J.na * J.nb;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < J.nchunks; ++c) s += J.part[(long long)c * tot + e];
        const int i = e / J.nb, j = e - i * J.nb;
        J.out[i + j * J.na] = (float)s;
    }
}

__global__ void __launch_bounds__(RR_THREADS) k_svdsmall(const ssa_svd_job* __restrict__ jobs) {
    extern __shared__ double dsm[];
    double* A = dsm;                    // column j of M at A + j * SLD
    double* Z = dsm + SSA_MAX_KP * SLD;
    __shared__ double nrm[SSA_MAX_KP];
    __shared__ int order[SSA_MAX_KP];
    __shared__ int notconv;
    const ssa_svd_job J = jobs[blockIdx.x];
    const int n = J.n;
    if (n < 1 || n > SSA_MAX_KP || J.nchunks < 1) {
        if (threadIdx.x == 0) check_fail(7, 1, (unsigned)n);
        return;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < J.nchunks; ++c) s += J.part[(long long)c * n * n + e];
        const int i = e / n, j = e - i * n;
        A[j * SLD + i] = s;
    }
    for (int c = warp; c < n; c += nw)
        for (int r = lane; r < n; r += 32) Z[c * SLD + r] = (r == c) ? 1.0 : 0.0;
    __syncthreads();
    onesided_jacobi(A, Z, n, &notconv, nrm);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {  // descending singular value
        const double v = nrm[i];
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const double w = nrm[j];
            rank += (w > v) || (w == v && j < i);
        }
        order[rank] = i;
    }
    __syncthreads();
    for (int j = warp; j < n; j += nw) {
        const int col = order[j];
        if (col < 0 || col >= n) {
            if (lane == 0) check_fail(7, 2, (unsigned)col);
            continue;
        }
        const double sg = nrm[col];
        const double isg = sg > 1e-300 ? 1.0 / sg : 0.0;
        for (int i = lane; i < n; i += 32) {
            J.Us[i + j * n] = (float)(A[col * SLD + i] * isg);
            J.Vs[i + j * n] = (float)Z[col * SLD + i];
            J.Dinv[i + j * n] = (i == j) ? (float)(sg > 1e-12 ? 1.0 / sg : 1.0) : 0.f;
        }
        if (lane == 0) {
            J.sigma[j] = sg;
            if (!isfinite(sg) && J.status) atomicOr(J.status, 2);
        }
    }
}

__global__ void __launch_bounds__(256) k_sortsign(const ssa_sortsign_job* __restrict__ jobs) {
    __shared__ double colsum[SSA_MAX_KP];
    __shared__ double sv[SSA_MAX_KP];
    __shared__ int pm[SSA_MAX_KP];
    const ssa_sortsign_job J = jobs[blockIdx.x];
    const int k = J.k;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (k < 1 || k > SSA_MAX_KP) {
        if (threadIdx.x == 0) check_fail(8, 1, (unsigned)k);
        return;
    }
    for (int c = warp; c < k; c += nw) {
        double s = 0.0;
        for (int r = lane; r < J.L; r += 32) s += (double)J.U[(long long)r + (long long)c * J.ldU];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) colsum[c] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < k; ++i) {
            sv[i] = J.sigma[i];
            pm[i] = i;
        }
        // the reference's exchange sort (MKL/ssa_opt.h:1896-1908)
        for (int i = 0; i < k - 1; ++i)
            for (int j = i + 1; j < k; ++j)
                if (sv[j] > sv[i]) {
                    const double t = sv[i];
                    sv[i] = sv[j];
                    sv[j] = t;
                    const int u = pm[i];
                    pm[i] = pm[j];
                    pm[j] = u;
                }
        for (int i = 0; i < k; ++i) {
            J.sigma[i] = sv[i];
            J.perm[i] = pm[i];
            J.sign[i] = (i >= J.sign_from && colsum[pm[i]] < 0.0) ? -1.f : 1.f;
        }
    }
}

__global__ void k_permcols(const ssa_permcols_job* __restrict__ jobs) {
    const ssa_permcols_job J = jobs[blockIdx.z];
    const int j = blockIdx.y;
    if (j >= J.k) return;
    const int src = J.perm[j];
    const float sg = J.sign[j];
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < J.m; r += gridDim.x * blockDim.x)
        J.dst[(long long)r + (long long)j * J.ldd] = sg * J.src[(long long)r + (long long)src * J.lds];
}

// ---------------------------------------------------------------------------------------------
// Small elementwise / reduction kernels (MSSA channel sums, contributions, Cadzow)
// ---------------------------------------------------------------------------------------------

__global__ void k_slabsum(float* out, const float* in, long long stride, int nslab, long long n, long long inst_stride) {
    // instance blockIdx.y: its nslab slabs start at in + y * inst_stride, its sum at out + y * inst_stride
    out += (long long)blockIdx.y * inst_stride;
    in += (long long)blockIdx.y * inst_stride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float acc = 0.f;
        for (int sl = 0; sl < nslab; ++sl) acc += in[(long long)sl * stride + i];
        out[i] = acc;
    }
}

__global__ void k_colnorm2(const float* A, long long sstride, long long ld, int m, int k, double* out) {
    __shared__ double red[32];
    const int s = blockIdx.y, j = blockIdx.x;
    const float* a = A + (long long)s * sstride + (long long)j * ld;
    double acc = 0.0;
    for (int r = threadIdx.x; r < m; r += blockDim.x) acc += (double)a[r] * (double)a[r];
    acc = block_sum<double>(acc, red);
    if (threadIdx.x == 0) out[(long long)s * k + j] = acc;
}

__global__ void k_diffnorm(const double* a, const double* b, long long n, double* out2) {
    // one CTA per vector: vector blockIdx.x at a + x n, b + x n, its two sums at out2 + 2 x
    a += (long long)blockIdx.x * n;
    b += (long long)blockIdx.x * n;
    out2 += 2 * (long long)blockIdx.x;
    __shared__ double red[32];
    double d2 = 0.0, a2 = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        const double d = a[i] - b[i];
        d2 += d * d;
        a2 += a[i] * a[i];
    }
    d2 = block_sum<double>(d2, red);
    a2 = block_sum<double>(a2, red);
    if (threadIdx.x == 0) {
        out2[0] = d2;
        out2[1] = a2;
    }
}

// Gap filling step: the reconstruction replaces the signal at the gap positions idx[0, n); out2 =
// {sum (new - old)^2, sum old^2} over the gaps (one CTA).
__global__ void k_gapupdate(double* x, const double* recon, const int* idx, int n, double* out2) {
    __shared__ double red[32];
    double d2 = 0.0, o2 = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int j = idx[i];
        const double nv = recon[j], ov = x[j];
        d2 += (nv - ov) * (nv - ov);
        o2 += ov * ov;
        x[j] = nv;
    }
    d2 = block_sum<double>(d2, red);
    o2 = block_sum<double>(o2, red);
    if (threadIdx.x == 0) {
        out2[0] = d2;
        out2[1] = o2;
    }
}

__global__ void __launch_bounds__(256) k_copy_segments(const ssa_copy_seg* __restrict__ segs) {
    const ssa_copy_seg S = segs[blockIdx.x];
    for (long long i = threadIdx.x; i < S.n; i += blockDim.x) S.dst[i] = S.src[i];
}

__global__ void k_axpby(const double* a, const double* b, double* out, double alpha, double beta, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = alpha * a[i] + beta * b[i];
}

// ---------------------------------------------------------------------------------------------
// W-correlation finish and LRF forecast
// ---------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(SMALL_THREADS) k_wfin(const ssa_wfin_job* __restrict__ jobs) {
    __shared__ double G[SSA_MAX_KP * SLD];
    const ssa_wfin_job J = jobs[blockIdx.x];
    const int k = J.k;
    reduce_packed(J.part, J.nchunks, k, G);
    __syncthreads();
    for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
        const int i = e / k, j = e % k;
        const double ni = sqrt(G[i * SLD + i]), nj = sqrt(G[j * SLD + j]);
        double w = 0.0;
        if (ni > 1e-12 && nj > 1e-12) w = G[i * SLD + j] / (ni * nj);
        J.W[e] = w;
    }
}

__global__ void __launch_bounds__(SMALL_THREADS) k_lrf(const ssa_lrf_job* __restrict__ jobs) {
    __shared__ double red[32];
    __shared__ double pi_s[SSA_MAX_KP];
    __shared__ int ok;
    const ssa_lrf_job J = jobs[blockIdx.x];
    const int L = J.L, ng = J.n_group;
    if (threadIdx.x == 0) {
        double nu2 = 0.0;
        for (int g = 0; g < ng; ++g) {
            const double p = (double)J.U[(long long)(L - 1) + (long long)J.group[g] * J.ld];
            pi_s[g] = p;
            nu2 += p * p;
        }
        *J.verticality = nu2;
        ok = nu2 < 1.0 - 1e-10;
        if (!ok) atomicOr(J.status, 4);
        red[0] = nu2;
    }
    __syncthreads();
    if (!ok) return;
    const double scale = 1.0 / (1.0 - red[0]);
    __syncthreads();
    const int w = L - 1;
    for (int j = threadIdx.x; j < w; j += blockDim.x) {
        double s = 0.0;
        for (int g = 0; g < ng; ++g) s += pi_s[g] * (double)J.U[(long long)j + (long long)J.group[g] * J.ld];
        J.R[j] = s * scale;
        J.buf[j] = J.recon[J.N - w + j];
    }
    __syncthreads();
    for (int h = 0; h < J.h; ++h) {
        double s = 0.0;
        for (int j = threadIdx.x; j < w; j += blockDim.x) s += J.R[j] * J.buf[h + j];
        s = block_sum<double>(s, red);
        if (threadIdx.x == 0) {
            J.buf[w + h] = s;
            J.out[h] = s;
        }
        __syncthreads();
    }
}

// Recurrence of the R-forecast from stored coefficients; forecasts so far stay in shared memory.
__global__ void __launch_bounds__(SMALL_THREADS) k_forecast_apply(const ssa_fc_job* __restrict__ jobs) {
    __shared__ double red[32];
    __shared__ double fo[SSA_FC_MAX_H];
    const ssa_fc_job J = jobs[blockIdx.x];
    const int w = J.w;
    for (int t = 0; t < J.h; ++t) {
        double s = 0.0;
        for (int j = threadIdx.x; j < w; j += blockDim.x) {
            const int i = t + j;
            s += J.R[j] * (i < w ? J.tail[i] : fo[i - w]);
        }
        s = block_sum<double>(s, red);
        if (threadIdx.x == 0) fo[t] = s;
        __syncthreads();
    }
    for (int t = threadIdx.x; t < J.h; t += blockDim.x) J.out[t] = fo[t];
}

__global__ void k_group_sum(ssa_gsum_job J) {
    const int s = blockIdx.z, g = blockIdx.y;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= J.N) return;
    const float* base = J.recon + (long long)s * J.recon_series;
    double acc = 0.0;
    for (int e = J.group_off[g]; e < J.group_off[g + 1]; ++e) {
        const int i = J.group_idx[e];
        if (i < 0 || i >= J.k) continue;
        acc += (double)base[(long long)i * J.ld_recon + t];
    }
    J.out[(long long)s * J.out_series + (long long)g * J.N + t] = acc;
}

__global__ void k_gaussian(float* out, long long ld, int rows, int ncols, int col0, unsigned long long seed) {
    const int c = blockIdx.y;
    const int npairs = (rows + 1) / 2;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npairs; i += gridDim.x * blockDim.x) {
        const float2 v = gauss_pair(seed, col0 + c, i);
        out[(long long)c * ld + 2 * i] = v.x;
        if (2 * i + 1 < rows) out[(long long)c * ld + 2 * i + 1] = v.y;
    }
}

// ---------------------------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------------------------

extern "C" int ssad_logh_for(int N) {
    int logm = 5;  // M >= 32
    while ((1 << logm) < N) ++logm;
    return logm - 1;
}

extern "C" int ssad_fft_h(int code) {
    if (code >= 4 && code <= SSA_MAX_LOGH_ALL) return 1 << code;
    if (code == SSA_FFT_3x13) return 3 << 13;
    if (code == SSA_FFT_3x14) return 3 << 14;
    if (code == SSA_FFT_5x13) return 5 << 13;
    return 0;
}

extern "C" int ssad_fft_code_for(int N) {
    const int logh = ssad_logh_for(N);
    if (logh > SSA_MAX_LOGH_ALL) return -1;  // beyond the largest length
    // between the cluster powers of two, the 3 * 2^a length when it suffices
    if (logh == 15 && N <= 2 * (3 << 13)) return SSA_FFT_3x13;
    if (logh == 16 && N <= 2 * (5 << 13)) return SSA_FFT_5x13;
    if (logh == 16 && N <= 2 * (3 << 14)) return SSA_FFT_3x14;
    return logh;
}

extern "C" int ssad_init_device(void) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    // one upload per device and process; the lock keeps two threads that make their first call
    // on the same device at once from uploading twice (the second would rewrite the tables while
    // the first one's kernels may already read them)
    static std::mutex mu;
    static bool done[64] = {false};
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 64 && done[dev]) return 0;
    std::vector<float2> tw(SSA_TW_N);
    for (int t = 0; t < SSA_TW_N; ++t) {
        const double a = -2.0 * M_PI * (double)t / (double)SSA_TW_N;
        tw[t] = make_float2((float)cos(a), (float)sin(a));
    }
    e = cudaMemcpyToSymbol(g_tw, tw.data(), sizeof(float2) * SSA_TW_N);
    if (e != cudaSuccess) return (int)e;
    std::vector<float2> tw3(SSA_TW3_N);
    for (int t = 0; t < SSA_TW3_N; ++t) {
        const double a = -2.0 * M_PI * (double)t / (double)SSA_TW3_N;
        tw3[t] = make_float2((float)cos(a), (float)sin(a));
    }
    e = cudaMemcpyToSymbol(g_tw3, tw3.data(), sizeof(float2) * SSA_TW3_N);
    if (e != cudaSuccess) return (int)e;
    std::vector<float2> tw5(SSA_TW5_N);
    for (int t = 0; t < SSA_TW5_N; ++t) {
        const double a = -2.0 * M_PI * (double)t / (double)SSA_TW5_N;
        tw5[t] = make_float2((float)cos(a), (float)sin(a));
    }
    e = cudaMemcpyToSymbol(g_tw5, tw5.data(), sizeof(float2) * SSA_TW5_N);
    if (e != cudaSuccess) return (int)e;
    if (dev < 64) done[dev] = true;
    return 0;
}

template <int LOGH>
static int smem_bytes(int bufs) { return fft_smem_f2<LOGH>(bufs) * (int)sizeof(float2); }

template <typename KernelT>
static cudaError_t set_smem(KernelT kern, int bytes) {
    if (bytes > 48 * 1024) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return cudaSuccess;
}

#define SSA_LOGH_DISPATCH(logh, CALL)                                    \
    switch (logh) {                                                      \
        case 4: CALL(4); break;                                          \
        case 5: CALL(5); break;                                          \
        case 6: CALL(6); break;                                          \
        case 7: CALL(7); break;                                          \
        case 8: CALL(8); break;                                          \
        case 9: CALL(9); break;                                          \
        case 10: CALL(10); break;                                        \
        case 11: CALL(11); break;                                        \
        case 12: CALL(12); break;                                        \
        case 13: CALL(13); break;                                        \
        case 14: CALL(14); break;                                        \
        default: return (int)cudaErrorInvalidValue;                      \
    }

template <int LOGH>
static int launch_spectrum(const ssa_col_job* jobs, int njobs, int maxcols, cudaStream_t st) {
    const int sm = smem_bytes<LOGH>(1);
    cudaError_t e = set_smem(k_spectrum<LOGH>, sm);
    if (e != cudaSuccess) return (int)e;
    k_spectrum<LOGH><<<dim3(maxcols, njobs), FftShape<LOGH>::BLOCK, sm, st>>>(jobs);
    return launched(cudaGetLastError());
}
template <int LOGH>
static int launch_corr(const ssa_col_job* jobs, int njobs, int maxcols, cudaStream_t st,
                       const ssa_tile* tiles = nullptr) {
    const int sm = smem_bytes<LOGH>(1);
    cudaError_t e = set_smem(k_corr<LOGH>, sm);
    if (e != cudaSuccess) return (int)e;
    const dim3 grid = tiles ? dim3(njobs, 1) : dim3(maxcols, njobs);  // tiles: njobs = tile count
    k_corr<LOGH><<<grid, FftShape<LOGH>::BLOCK, sm, st>>>(jobs, tiles, njobs);
    return launched(cudaGetLastError());
}
template <int LOGH>
static int launch_corr_spec(const ssa_col_job* jobs, int njobs, int maxcols, cudaStream_t st) {
    const int sm = smem_bytes<LOGH>(1);
    cudaError_t e = set_smem(k_corr_spec<LOGH>, sm);
    if (e != cudaSuccess) return (int)e;
    k_corr_spec<LOGH><<<dim3(maxcols, njobs), FftShape<LOGH>::BLOCK, sm, st>>>(jobs);
    return launched(cudaGetLastError());
}
template <int LOGH>
static int launch_corr_acc(const ssa_col_job* jobs, int njobs, int maxcols, int first, cudaStream_t st) {
    const int sm = smem_bytes<LOGH>(1);
    cudaError_t e = set_smem(k_corr_acc<LOGH>, sm);
    if (e != cudaSuccess) return (int)e;
    k_corr_acc<LOGH><<<dim3(maxcols, njobs), FftShape<LOGH>::BLOCK, sm, st>>>(jobs, first);
    return launched(cudaGetLastError());
}
template <int LOGH>
static int launch_elem(const ssa_col_job* jobs, int njobs, int maxcols, cudaStream_t st) {
    const int sm = smem_bytes<LOGH>(2);
    if (sm > 227 * 1024) return (int)cudaErrorInvalidValue;
    cudaError_t e = set_smem(k_elem_recon<LOGH>, sm);
    if (e != cudaSuccess) return (int)e;
    k_elem_recon<LOGH><<<dim3(maxcols, njobs), FftShape<LOGH>::BLOCK, sm, st>>>(jobs);
    return launched(cudaGetLastError());
}
template <int LOGH>
static int launch_elem1(const ssa_col_job* jobs, int njobs, int maxcols, cudaStream_t st) {
    const int sm = smem_bytes<LOGH>(1);
    cudaError_t e = set_smem(k_elem_recon1<LOGH>, sm);
    if (e != cudaSuccess) return (int)e;
    k_elem_recon1<LOGH><<<dim3(maxcols, njobs), FftShape<LOGH>::BLOCK, sm, st>>>(jobs);
    return launched(cudaGetLastError());
}
template <int LOGH>
static int launch_recon(const ssa_recon_job* jobs, int njobs, cudaStream_t st) {
    const int sm = smem_bytes<LOGH>(1);
    cudaError_t e = set_smem(k_recon<LOGH>, sm);
    if (e != cudaSuccess) return (int)e;
    k_recon<LOGH><<<dim3(1, njobs), FftShape<LOGH>::BLOCK, sm, st>>>(jobs);
    return launched(cudaGetLastError());
}

// Real FFT length 32768 (logh 14) on 2-CTA clusters of 8192-point CTAs (1) instead of one CTA of
// 1024 threads (0, the default); a per-bucket choice of the autotuner.
static int g_cl14 = 0;
extern "C" void ssad_set_cl14(int on) { g_cl14 = on != 0; }
extern "C" int ssad_cl14(void) { return g_cl14; }

#include "ssa_cluster.cuh"
#include "ssa_tc.cuh"

static int g_wcorr_tc = -1;  // -1: not yet read from the environment

extern "C" void ssad_set_wcorr_tc(int mode) { g_wcorr_tc = (mode >= 0 && mode <= 3) ? mode : 1; }

extern "C" int ssad_wcorr_tc(void) {
    if (g_wcorr_tc < 0) {
        const char* v = getenv("SSA_WCORR_FP64");
        g_wcorr_tc = (v && v[0] == '1') ? 0 : 1;
    }
    return g_wcorr_tc;
}

// Row products of the randomized pipelines on the tensor cores (1) or on the CUDA cores (0, the
// default: measured faster on the mixed stream, the tensor-core form being bound by the latency
// of its register-staged row loads).
// SSA_ROWMUL_TC=1 in the environment selects the tensor-core form at start-up.
static int g_rowmul_tc = -1;  // -1: not yet read from the environment
extern "C" void ssad_set_rowmul_tc(int on) { g_rowmul_tc = on != 0; }
extern "C" int ssad_rowmul_tc_on(void) {
    if (g_rowmul_tc < 0) {
        const char* v = getenv("SSA_ROWMUL_TC");
        g_rowmul_tc = (v && v[0] == '1') ? 1 : 0;
    }
    return g_rowmul_tc;
}

extern "C" int ssad_rowmul_tc(const ssa_rowmul_job* d_jobs, int njobs, int maxrows, int maxn, void* stream) {
    if (njobs <= 0 || maxrows <= 0) return 0;
    if (maxn > SSA_MAX_KP) return (int)cudaErrorInvalidValue;
    return launch_rowmul_tc(d_jobs, njobs, maxrows, (cudaStream_t)stream);
}

extern "C" int ssad_gram_tc(const ssa_wgram_job* d_jobs, int njobs, int maxchunks, void* stream) {
    if (njobs <= 0 || maxchunks <= 0) return 0;
    const int mode = ssad_wcorr_tc();
    return launch_gram_tc(d_jobs, njobs, maxchunks, mode == 0 ? 1 : mode, (cudaStream_t)stream);
}

extern "C" int ssad_spectrum(const ssa_col_job* d_jobs, int njobs, int maxcols, int logh, void* stream) {
    if (njobs <= 0 || maxcols <= 0) return 0;
    if (logh > SSA_MAX_LOGH || (logh == 14 && g_cl14))  // 15-19, and 14 on 2-CTA clusters when selected
        return cl_col_dispatch(CL_SPEC, d_jobs, njobs, maxcols, logh, (cudaStream_t)stream);
#define CALL(L) return launch_spectrum<L>(d_jobs, njobs, maxcols, (cudaStream_t)stream)
    SSA_LOGH_DISPATCH(logh, CALL)
#undef CALL
    return 0;
}
extern "C" int ssad_multi_tile_cols(int logh) {
    return (logh >= SSA_MULTI_MIN_LOGH && logh <= SSA_MULTI_MAX_LOGH) ? 1 << (SSA_MULTI_MAX_LOGH - logh) : 0;
}
extern "C" int ssad_corr_multi(const ssa_col_job* d_jobs, const ssa_tile* d_tiles, int ntiles, int* d_head, int nctas,
                               void* stream) {
    if (ntiles <= 0) return 0;
    const int sm = multi_smem_f2() * (int)sizeof(float2);
    cudaError_t e = set_smem(k_corr_multi, sm);
    if (e != cudaSuccess) return (int)e;
    if (nctas <= 0) {
        int dev = 0, nsm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        nctas = 2 * (nsm > 0 ? nsm : 148);
    }
    if (nctas > ntiles) nctas = ntiles;
    k_corr_multi<<<nctas, 512, sm, (cudaStream_t)stream>>>(d_jobs, d_tiles, ntiles, d_head);
    return launched(cudaGetLastError());
}
extern "C" int ssad_corr(const ssa_col_job* d_jobs, int njobs, int maxcols, int logh, void* stream) {
    if (njobs <= 0 || maxcols <= 0) return 0;
    if (logh > SSA_MAX_LOGH || (logh == 14 && g_cl14))  // 15-19, and 14 on 2-CTA clusters when selected
        return cl_col_dispatch(CL_CORR, d_jobs, njobs, maxcols, logh, (cudaStream_t)stream);
#define CALL(L) return launch_corr<L>(d_jobs, njobs, maxcols, (cudaStream_t)stream)
    SSA_LOGH_DISPATCH(logh, CALL)
#undef CALL
    return 0;
}
extern "C" int ssad_corr_tiles(const ssa_col_job* d_jobs, const ssa_tile* d_tiles, int ntiles, int logh, void* stream) {
    if (ntiles <= 0) return 0;
    if (logh > SSA_MAX_LOGH || (logh == 14 && g_cl14))
        return cl_col_dispatch(CL_CORR, d_jobs, ntiles, 1, logh, (cudaStream_t)stream, d_tiles);
#define CALL(L) return launch_corr<L>(d_jobs, ntiles, 1, (cudaStream_t)stream, d_tiles)
    SSA_LOGH_DISPATCH(logh, CALL)
#undef CALL
    return 0;
}
extern "C" int ssad_corr_spec(const ssa_col_job* d_jobs, int njobs, int maxcols, int logh, void* stream) {
    if (njobs <= 0 || maxcols <= 0) return 0;
#define CALL(L) return launch_corr_spec<L>(d_jobs, njobs, maxcols, (cudaStream_t)stream)
    SSA_LOGH_DISPATCH(logh, CALL)
#undef CALL
    return 0;
}
extern "C" int ssad_corr_acc(const ssa_col_job* d_jobs, int njobs, int maxcols, int logh, int first, void* stream) {
    if (njobs <= 0 || maxcols <= 0) return 0;
#define CALL(L) return launch_corr_acc<L>(d_jobs, njobs, maxcols, first, (cudaStream_t)stream)
    SSA_LOGH_DISPATCH(logh, CALL)
#undef CALL
    return 0;
}
extern "C" int ssad_elem_recon(const ssa_col_job* d_jobs, int njobs, int maxcols, int logh, void* stream) {
    if (njobs <= 0 || maxcols <= 0) return 0;
#define CALL(L) return launch_elem<L>(d_jobs, njobs, maxcols, (cudaStream_t)stream)
    SSA_LOGH_DISPATCH(logh, CALL)
#undef CALL
    return 0;
}
extern "C" int ssad_elem_recon1(const ssa_col_job* d_jobs, int njobs, int maxcols, int logh, void* stream) {
    if (njobs <= 0 || maxcols <= 0) return 0;
    if (logh > SSA_MAX_LOGH || (logh == 14 && g_cl14))  // 15-19, and 14 on 2-CTA clusters when selected
        return cl_col_dispatch(CL_ELEM, d_jobs, njobs, maxcols, logh, (cudaStream_t)stream);
#define CALL(L) return launch_elem1<L>(d_jobs, njobs, maxcols, (cudaStream_t)stream)
    SSA_LOGH_DISPATCH(logh, CALL)
#undef CALL
    return 0;
}
extern "C" int ssad_group_sum_ragged(const ssa_rgsum_job* d_jobs, int njobs, int maxN, const int* group_idx,
                                     const int* group_off, int n_groups, void* stream) {
    if (njobs <= 0 || n_groups <= 0 || maxN <= 0) return 0;
    if (njobs > 65535 || n_groups > 65535) return (int)cudaErrorInvalidValue;
    k_group_sum_ragged<<<dim3((maxN + 255) / 256, n_groups, njobs), 256, 0, (cudaStream_t)stream>>>(d_jobs, group_idx,
                                                                                                    group_off);
    return launched(cudaGetLastError());
}
extern "C" int ssad_recon(const ssa_recon_job* d_jobs, int njobs, int logh, void* stream) {
    if (njobs <= 0) return 0;
    if (logh > SSA_MAX_LOGH) return cl_recon_dispatch(d_jobs, njobs, logh, (cudaStream_t)stream);
#define CALL(L) return launch_recon<L>(d_jobs, njobs, (cudaStream_t)stream)
    SSA_LOGH_DISPATCH(logh, CALL)
#undef CALL
    return 0;
}

extern "C" int ssad_gram(const ssa_gram_job* d_jobs, int njobs, int maxchunks, int weighted, void* stream) {
    if (njobs <= 0 || maxchunks <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = weighted ? set_smem(k_gram<true>, GRAM_SMEM) : set_smem(k_gram<false>, GRAM_SMEM);
    if (e != cudaSuccess) return (int)e;
    if (weighted)
        k_gram<true><<<dim3(maxchunks, njobs), GRAM_MMA_THREADS, GRAM_SMEM, st>>>(d_jobs);
    else
        k_gram<false><<<dim3(maxchunks, njobs), GRAM_MMA_THREADS, GRAM_SMEM, st>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_chol(const ssa_chol_job* d_jobs, int njobs, void* stream) {
    if (njobs <= 0) return 0;
    cudaError_t e = set_smem(k_chol, SMALL_SMEM);
    if (e != cudaSuccess) return (int)e;
    k_chol<<<njobs, SMALL_THREADS, SMALL_SMEM, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_rowmul(const ssa_rowmul_job* d_jobs, int njobs, int maxrows, int maxn, void* stream) {
    if (njobs <= 0 || maxrows <= 0) return 0;
    if (maxn > SSA_MAX_KP) return (int)cudaErrorInvalidValue;
    cudaError_t e = set_smem(k_rowmul, RM_SMEM);
    if (e != cudaSuccess) return (int)e;
    k_rowmul<<<dim3((maxrows + RM_ROWS - 1) / RM_ROWS, njobs), RM_THREADS, RM_SMEM, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_rr(const ssa_rr_job* d_jobs, int njobs, void* stream) {
    if (njobs <= 0) return 0;
    cudaError_t e = set_smem(k_rr, SMALL_SMEM);
    if (e != cudaSuccess) return (int)e;
    k_rr<<<njobs, RR_THREADS, SMALL_SMEM, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_wfin(const ssa_wfin_job* d_jobs, int njobs, void* stream) {
    if (njobs <= 0) return 0;
    k_wfin<<<njobs, SMALL_THREADS, 0, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_lrf(const ssa_lrf_job* d_jobs, int njobs, void* stream) {
    if (njobs <= 0) return 0;
    k_lrf<<<njobs, SMALL_THREADS, 0, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_forecast_apply(const ssa_fc_job* d_jobs, int njobs, void* stream) {
    if (njobs <= 0) return 0;
    k_forecast_apply<<<njobs, SMALL_THREADS, 0, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_group_sum(ssa_gsum_job job, void* stream) {
    if (job.B <= 0 || job.n_groups <= 0) return 0;
    k_group_sum<<<dim3((job.N + 255) / 256, job.n_groups, job.B), 256, 0, (cudaStream_t)stream>>>(job);
    return launched(cudaGetLastError());
}

extern "C" int ssad_xgram(const ssa_xgram_job* d_jobs, int njobs, int maxchunks, void* stream) {
    if (njobs <= 0 || maxchunks <= 0) return 0;
    cudaError_t e = set_smem(k_xgram, XG_SMEM);
    if (e != cudaSuccess) return (int)e;
    k_xgram<<<dim3(maxchunks, njobs), GRAM_THREADS, XG_SMEM, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_xreduce(const ssa_xreduce_job* d_jobs, int njobs, void* stream) {
    if (njobs <= 0) return 0;
    k_xreduce<<<njobs, 256, 0, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_svdsmall(const ssa_svd_job* d_jobs, int njobs, void* stream) {
    if (njobs <= 0) return 0;
    cudaError_t e = set_smem(k_svdsmall, SMALL_SMEM);
    if (e != cudaSuccess) return (int)e;
    k_svdsmall<<<njobs, RR_THREADS, SMALL_SMEM, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_sortsign(const ssa_sortsign_job* d_jobs, int njobs, void* stream) {
    if (njobs <= 0) return 0;
    k_sortsign<<<njobs, 256, 0, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_permcols(const ssa_permcols_job* d_jobs, int njobs, int maxrows, void* stream) {
    if (njobs <= 0 || maxrows <= 0) return 0;
    const int bx = min((maxrows + 255) / 256, 64);
    k_permcols<<<dim3(bx, SSA_MAX_KP, njobs), 256, 0, (cudaStream_t)stream>>>(d_jobs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_slabsum_batch(float* out, const float* in, long long stride, int nslab, long long n, int ninst,
                                  long long inst_stride, void* stream) {
    if (n <= 0 || nslab <= 0 || ninst <= 0) return 0;
    const long long blocks = (n + 255) / 256;
    const unsigned bx = (unsigned)(blocks < 4096 ? blocks : 4096);
    k_slabsum<<<dim3(bx, (unsigned)ninst), 256, 0, (cudaStream_t)stream>>>(out, in, stride, nslab, n, inst_stride);
    return launched(cudaGetLastError());
}
extern "C" int ssad_slabsum(float* out, const float* in, long long stride, int nslab, long long n, void* stream) {
    return ssad_slabsum_batch(out, in, stride, nslab, n, 1, 0, stream);
}

extern "C" int ssad_colnorm2(const float* A, long long sstride, long long ld, int m, int k, int nb, double* out,
                             void* stream) {
    if (nb <= 0 || k <= 0) return 0;
    k_colnorm2<<<dim3(k, nb), 256, 0, (cudaStream_t)stream>>>(A, sstride, ld, m, k, out);
    return launched(cudaGetLastError());
}

extern "C" int ssad_gapupdate(double* x, const double* recon, const int* idx, int n, double* out2, void* stream) {
    if (n < 1) return 0;
    k_gapupdate<<<1, 256, 0, (cudaStream_t)stream>>>(x, recon, idx, n, out2);
    return launched(cudaGetLastError());
}

extern "C" int ssad_copy_segments(const ssa_copy_seg* d_segs, int nseg, void* stream) {
    if (nseg <= 0) return 0;
    k_copy_segments<<<nseg, 256, 0, (cudaStream_t)stream>>>(d_segs);
    return launched(cudaGetLastError());
}

extern "C" int ssad_diffnorm(const double* a, const double* b, long long n, double* out2, void* stream) {
    k_diffnorm<<<1, 1024, 0, (cudaStream_t)stream>>>(a, b, n, out2);
    return launched(cudaGetLastError());
}
extern "C" int ssad_diffnorm_batch(const double* a, const double* b, long long n, int nvec, double* out2,
                                   void* stream) {
    if (nvec <= 0 || n <= 0) return 0;
    k_diffnorm<<<nvec, 1024, 0, (cudaStream_t)stream>>>(a, b, n, out2);
    return launched(cudaGetLastError());
}

extern "C" int ssad_axpby(const double* a, const double* b, double* out, double alpha, double beta, long long n,
                          void* stream) {
    if (n <= 0) return 0;
    const long long blocks = (n + 255) / 256;
    k_axpby<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, (cudaStream_t)stream>>>(a, b, out, alpha, beta, n);
    return launched(cudaGetLastError());
}

extern "C" int ssad_gaussian(float* out, long long ld, int rows, int ncols, int col0, unsigned long long seed,
                             void* stream) {
    if (rows <= 0 || ncols <= 0) return 0;
    const int npairs = (rows + 1) / 2;
    const int bx = (npairs + 255) / 256;
    k_gaussian<<<dim3(bx < 64 ? bx : 64, ncols), 256, 0, (cudaStream_t)stream>>>(out, ld, rows, ncols, col0, seed);
    return launched(cudaGetLastError());
}

// ---------------------------------------------------------------------------------------------
// W-correlation without any device allocation (ssa_wcorr_noalloc, declared in ssa_b200.h)
//
// Some callers cannot let a library allocate device memory: a host application whose device
// memory is owned up front by another framework's allocator (cudaMalloc behind its back would
// break its accounting), or a latency-critical loop that must not take cudaMalloc's implicit
// device synchronisation. This entry point serves them: it computes the W-correlation matrix of
// a decomposition the caller already holds in device memory, and the only device memory it
// touches besides the caller's inputs and output is the fixed array below, which every GPU that
// loads the library holds until the process exits.
// ---------------------------------------------------------------------------------------------

#define SSA_NOALLOC_JOB_BYTES 1024
#define SSA_NOALLOC_ROWS 1024  // Gram rows per partial
#define SSA_NOALLOC_NCH ((SSA_NOALLOC_MAX_N + SSA_NOALLOC_ROWS - 1) / SSA_NOALLOC_ROWS)
#define SSA_NOALLOC_PART_BYTES (SSA_NOALLOC_NCH * (SSA_NOALLOC_MAX_K * (SSA_NOALLOC_MAX_K + 1) / 2) * 8)
#define SSA_NOALLOC_RECON_BYTES (SSA_NOALLOC_MAX_K * SSA_NOALLOC_MAX_N * 4)
#define SSA_NOALLOC_BYTES (SSA_NOALLOC_JOB_BYTES + SSA_NOALLOC_PART_BYTES + SSA_NOALLOC_RECON_BYTES)

// Scratch shared by every call on a device: [job tables | Gram partials | reconstructions].
static __device__ __align__(256) unsigned char g_noalloc_scratch[SSA_NOALLOC_BYTES];

#include <cstring>

// The three job tables sit in 256-byte slots at the start of the scratch array.
static_assert(sizeof(ssa_col_job) <= 256, "ssa_col_job must fit its 256-byte scratch slot");
static_assert(sizeof(ssa_gram_job) <= 256, "ssa_gram_job must fit its 256-byte scratch slot");
static_assert(512 + sizeof(ssa_wfin_job) <= SSA_NOALLOC_JOB_BYTES, "ssa_wfin_job must fit the job area");

static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[64];
static bool g_noalloc_ready[64];

// Per-device set-up, run by the first call on a device with that device current: the library's
// own one-time device initialisation (twiddle tables, shared with every other entry point and
// done once per device), then the lookup of the scratch array's device address (host code must
// not pass the symbol itself to a kernel: on the host it is only a stand-in).
static int noalloc_setup(int dev, void** scratch) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ready[dev]) {
        *scratch = g_noalloc_ptr[dev];
        return 0;
    }
    if (ssad_init_device() != 0) return -1;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return -1;
    g_noalloc_ptr[dev] = p;
    g_noalloc_ready[dev] = true;
    *scratch = p;
    return 0;
}

// Stores the three job tables into their scratch slots. They travel as kernel parameters, which
// the launch copies, so the call neither stages host memory nor waits on the stream.
__global__ void k_noalloc_jobs(ssa_col_job je, ssa_gram_job jg, ssa_wfin_job jw, ssa_col_job* de,
                               ssa_gram_job* dg, ssa_wfin_job* dw) {
    *de = je;
    *dg = jg;
    *dw = jw;
}

extern "C" __attribute__((visibility("default"))) int ssa_wcorr_noalloc(
    const float* d_U, long long ldU, const float* d_V, long long ldV, const double* d_sigma, int N, int L, int k,
    double* d_W, void* stream) {
    if (!d_U || !d_V || !d_sigma || !d_W || N < 4 || L < 2 || L > N - 1 || k < 1) return -1;
    const int K = N - L + 1;
    if (k > L || k > K || ldU < L || ldV < K || (ldU & 1) || (ldV & 1) ||
        (((uintptr_t)d_U) & 7) || (((uintptr_t)d_V) & 7))
        return -1;
    if (N > SSA_NOALLOC_MAX_N || k > SSA_NOALLOC_MAX_K) return -2;  // beyond the fixed scratch
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
    void* scratch = nullptr;
    if (noalloc_setup(dev, &scratch) != 0) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char* base = (unsigned char*)scratch;
    ssa_col_job* d_elem = (ssa_col_job*)base;
    ssa_gram_job* d_gram = (ssa_gram_job*)(base + 256);
    ssa_wfin_job* d_wfin = (ssa_wfin_job*)(base + 512);
    double* d_part = (double*)(base + SSA_NOALLOC_JOB_BYTES);
    float* d_recon = (float*)(base + SSA_NOALLOC_JOB_BYTES + SSA_NOALLOC_PART_BYTES);
    const long long ldN = (N + 3) & ~3LL;
    const int nch = (N + SSA_NOALLOC_ROWS - 1) / SSA_NOALLOC_ROWS;
    // Every partial and every reconstruction row the later stages read is written first, so the
    // scratch needs no clearing between calls.
    ssa_col_job je;
    memset(&je, 0, sizeof(je));
    je.in = d_U;
    je.ld_in = ldU;
    je.n_in = L;
    je.in2 = d_V;
    je.ld_in2 = ldV;
    je.n_in2 = K;
    je.scale = d_sigma;
    je.out = d_recon;
    je.ld_out = ldN;
    je.ncols = k;
    je.N = N;
    je.L = L;
    je.K = K;
    ssa_gram_job jg;
    memset(&jg, 0, sizeof(jg));
    jg.A = d_recon;
    jg.part = d_part;
    jg.ld = ldN;
    jg.m = N;
    jg.n = k;
    jg.rows_per_cta = SSA_NOALLOC_ROWS;
    jg.weighted = 1;
    jg.N = N;
    jg.L = L;
    jg.K = K;
    ssa_wfin_job jw;
    memset(&jw, 0, sizeof(jw));
    jw.part = d_part;
    jw.W = d_W;
    jw.nchunks = nch;
    jw.k = k;
    k_noalloc_jobs<<<1, 1, 0, st>>>(je, jg, jw, d_elem, d_gram, d_wfin);
    if (launched(cudaGetLastError()) != 0) return -1;
    if (ssad_elem_recon(d_elem, 1, k, ssad_logh_for(N), st) != 0) return -1;
    if (ssad_gram(d_gram, 1, nch, 1, st) != 0) return -1;
    if (ssad_wfin(d_wfin, 1, st) != 0) return -1;
    return 0;
}
