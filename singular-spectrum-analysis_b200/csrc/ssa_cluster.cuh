// FFT lengths beyond one CTA's shared memory: each transform runs on a thread-block cluster of
// C CTAs of H1 = 8192 points, H = C H1 complex points (real length M = 2H): C = 4 and 8 for
// M = 2^16 and 2^17, C = 3, 5 and 6 for M = 3 * 2^14, 5 * 2^14 and 3 * 2^15, which cut the
// padding of the series between the powers of two (series up to N = 131072).
//
// Packed sequence z[n] = a[2n] + i a[2n+1], n < H = C H1 (H1 = 8192). CTA r of the cluster holds
// the decimated sequence z_r[m] = z[C m + r] and transforms it locally (fft_block, H1 points):
// Z_r = DFT_H1(z_r). The H-point spectrum is then
//     Z[k1 + H1 k2] = sum_r W_H^{r k1} W_C^{r k2} Z_r[k1],   k1 < H1, k2 < C,
// a C-point DFT per k1 of the twiddled partial spectra. Each k1 and its mirror H1 - k1 belong to
// one CTA (the real-FFT unpacking pairs bin k with H - k, and H - (k1 + H1 k2) =
// (H1 - k1) + H1 (C - 1 - k2)), which reads the C partial values at both through distributed
// shared memory, forms the 2C bins, applies the per-kernel spectral operation and, where an
// inverse transform follows, writes the inverse combination
//     T_r[k1] = W_H^{-r k1} sum_k2 Z'[k1 + H1 k2] W_C^{-r k2}
// back into CTA r's buffer at the same slot k1 (only the owner of k1 touches slot k1 in any
// CTA, so reading and writing in place needs no barrier in between). After a cluster barrier
// each CTA inverts its T_r locally: z'[C m + r] = IDFT_H1(T_r)[m].
//
// Cluster barriers: one after the local forward transforms (every partial spectrum complete and
// every CTA resident), one after the exchange; a kernel whose last remote access is a read
// (spectrum) or a write into rank 0 (norm reduction) ends with one more, so that no CTA leaves
// while another still addresses its shared memory.

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

// 8192-point CTAs, two per SM (16384-point CTAs, one per SM, measured 1.3% slower)
#define SSA_CL_LOGH1 13
#define SSA_CL_MAX_LOGH 16

__host__ __device__ constexpr int cl_ilog2(int v) { return v <= 1 ? 0 : 1 + cl_ilog2(v >> 1); }

template <int C_>
struct ClShape {
    static constexpr int LOGH1 = SSA_CL_LOGH1;
    static constexpr int H1 = 1 << LOGH1;
    static constexpr int C = C_;
    static constexpr int H = C * H1;
    static constexpr int BLOCK = FftShape<LOGH1>::BLOCK;
    static constexpr int MINB = BLOCK >= 1024 ? 1 : 2;  // CTAs per SM the kernels are built for
    static constexpr bool POW2 = (C & (C - 1)) == 0;
    static constexpr bool FIVE = C == 5;
    static_assert(POW2 || C % 3 == 0 || FIVE, "cluster sizes are 2^a, 3 * 2^a or 5");
    // twiddle table of resolution M = 2H: 2^LOGM, 3 * 2^A3 or 5 * 2^A5
    static constexpr int LOGM = cl_ilog2(2 * H);
    static constexpr int A3 = cl_ilog2(2 * H / 3);
    static constexpr int A5 = cl_ilog2(2 * H / 5);
    using Tw = typename std::conditional<
        POW2, TwSplit<(POW2 ? LOGM : 1)>,
        typename std::conditional<FIVE, TwSplit5<(FIVE ? A5 : 9)>, TwSplit3<(POW2 || FIVE ? 9 : A3)>>::type>::type;
};

template <int C>
__device__ __forceinline__ void cl_load_twM(float2* tab) {
    using S = ClShape<C>;
    if constexpr (S::POW2)
        load_twiddles<S::LOGM>(tab);
    else if constexpr (S::FIVE)
        load_twiddles5<S::A5>(tab);
    else
        load_twiddles3<S::A3>(tab);
}

template <int C>
__host__ __device__ constexpr int cl_smem_f2() {
    return spad_size(ClShape<C>::H1) + TwSplit<SSA_CL_LOGH1 + 1>::N + ClShape<C>::Tw::N;
}

enum { CL_SPEC = 0, CL_CORR = 1, CL_ELEM = 2, CL_RECON = 3 };

// Operands of the per-bin spectral operation.
struct ClOp {
    const float2* X;     // CL_CORR: signal spectrum (H + 1 bins)
    float2* spec;        // CL_SPEC: output spectrum
    const float2* us;    // CL_ELEM: spectrum of sigma u
    const ssa_recon_job* R;  // CL_RECON
};

// Sum over the group of Us_i[k] Vs_i[k] (CL_RECON).
__device__ __forceinline__ float2 cl_group_product(const ssa_recon_job& J, int k) {
    float2 p = make_float2(0.f, 0.f);
    for (int g = 0; g < J.n_group; ++g) {
        const int i = J.group[g];
        if (i < 0 || i >= J.k) continue;
        const float2* us = reinterpret_cast<const float2*>(J.Us + (long long)i * J.ld_spec);
        const float2* vs = reinterpret_cast<const float2*>(J.Vs + (long long)i * J.ld_spec);
        p = cadd(p, cmul(us[k], vs[k]));
    }
    return p;
}

// Bins k and H - k (1 <= k <= H/2) of the packed transform in zk, zm are replaced by the packed
// output spectrum (or, for CL_SPEC, the real spectrum is written out).
template <int C, int KIND>
__device__ __forceinline__ void cl_pair(const ClOp& op, int k, float2& zk, float2& zm, const float2* twM) {
    constexpr int H = ClShape<C>::H;
    const float2 w = twiddle_s<typename ClShape<C>::Tw, false>(twM, k);
    float2 pk, pm;
    if constexpr (KIND == CL_RECON) {
        pk = cl_group_product(*op.R, k);
        pm = cl_group_product(*op.R, H - k);
    } else {
        float2 ak, am;
        unpack_pair<0>(zk, zm, w, ak, am);
        if constexpr (KIND == CL_SPEC) {
            op.spec[k] = ak;
            op.spec[H - k] = am;
            return;
        } else if constexpr (KIND == CL_CORR) {
            pk = cmulc(op.X[k], ak);
            pm = cmulc(op.X[H - k], am);
        } else {
            pk = cmul(op.us[k], ak);
            pm = cmul(op.us[H - k], am);
        }
    }
    pack_pair(pk, pm, w, zk, zm);
}

// Bin 0 with the Nyquist bin H, both real, packed together in z0.
template <int C, int KIND>
__device__ __forceinline__ void cl_dc(const ClOp& op, float2& z0) {
    constexpr int H = ClShape<C>::H;
    float2 zk, zm;
    if constexpr (KIND == CL_SPEC) {
        op.spec[0] = make_float2(z0.x + z0.y, 0.f);
        op.spec[H] = make_float2(z0.x - z0.y, 0.f);
        return;
    } else if constexpr (KIND == CL_CORR) {
        pack_pair(cscale(op.X[0], z0.x + z0.y), cscale(op.X[H], z0.x - z0.y), make_float2(1.f, 0.f), zk, zm);
    } else if constexpr (KIND == CL_ELEM) {
        const float p0 = op.us[0].x * (z0.x + z0.y);
        const float ph = op.us[H].x * (z0.x - z0.y);
        pack_pair(make_float2(p0, 0.f), make_float2(ph, 0.f), make_float2(1.f, 0.f), zk, zm);
    } else {
        pack_pair(cl_group_product(*op.R, 0), cl_group_product(*op.R, H), make_float2(1.f, 0.f), zk, zm);
    }
    z0 = zk;
}

// Distributed shared memory through 32-bit shared::cluster addresses: the address of a slot in
// CTA q's buffer is mapped on the fly, so no per-rank 64-bit pointers stay live in registers.
__device__ __forceinline__ uint32_t cl_map(uint32_t local, int q) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(q));
    return r;
}
// The loads carry no memory clobber, so that the compiler may move the independent global loads
// of the spectral operation (signal spectrum bins) ahead of them; they stay ordered with the
// volatile stores below, and the cluster barriers around the exchange order them with every
// other access of the buffers.
__device__ __forceinline__ float2 cl_ld(uint32_t a) {
    float2 v;
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ void cl_st(uint32_t a, float2 v) {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}

// z[q] *= w^q (q = 1 .. C-1), or times conj(w)^q for the inverse; w^q by repeated products
// (about q ulp each, as the powers inside the radix-16 passes).
template <int C, bool INV>
__device__ __forceinline__ void cl_twiddle(float2* z, float2 w) {
    if (INV) w.y = -w.y;
    float2 wq = w;
#pragma unroll
    for (int q = 1; q < C; ++q) {
        z[q] = cmul(z[q], wq);
        if (q + 1 < C) wq = cmul(wq, w);
    }
}

// Owner phase over this CTA's items: gather (unless CL_RECON), spectral operation, scatter
// (unless CL_SPEC). sbase is the shared-window address of this CTA's transform buffer; the
// same offset in CTA q's window is CTA q's slot.
template <int C_, int KIND>
__device__ __forceinline__ void cl_exchange(uint32_t sbase, const float2* twM, int rank, const ClOp& op) {
    using S = ClShape<C_>;
    constexpr int C = S::C, H1 = S::H1, H = S::H;
    for (int g = rank * S::BLOCK + (int)threadIdx.x; g <= H1 / 2; g += C * S::BLOCK) {
        const int ka = g, kb = (H1 - g) & (H1 - 1);
        const bool self = ka == kb;  // k1 = 0 or H1/2
        const uint32_t aa = sbase + 8u * (uint32_t)spad(ka), ab = sbase + 8u * (uint32_t)spad(kb);
        float2 za[C], zb[C];
        // W_H^{q k1} for q = 1 .. C-1 as powers of one table value (lanes read consecutive
        // table entries; a lookup per power would stride the table by 2q entries)
        const float2 wa = twiddle_s<typename S::Tw, false>(twM, 2 * ka);
        const float2 wb = twiddle_s<typename S::Tw, false>(twM, 2 * kb);
        if constexpr (KIND != CL_RECON) {
#pragma unroll
            for (int q = 0; q < C; ++q) za[q] = cl_ld(cl_map(aa, q));
            cl_twiddle<C, false>(za, wa);
            dftR<C, false>(za);
            if (!self) {
#pragma unroll
                for (int q = 0; q < C; ++q) zb[q] = cl_ld(cl_map(ab, q));
                cl_twiddle<C, false>(zb, wb);
                dftR<C, false>(zb);
            }
        } else {
#pragma unroll
            for (int q = 0; q < C; ++q) za[q] = zb[q] = make_float2(0.f, 0.f);
        }
        if (!self) {
            // bin ka + H1 q pairs with kb + H1 (C - 1 - q)
#pragma unroll
            for (int q = 0; q < C; ++q) {
                const int k = ka + H1 * q;
                if (k <= H / 2) cl_pair<C_, KIND>(op, k, za[q], zb[C - 1 - q], twM);
                else cl_pair<C_, KIND>(op, H - k, zb[C - 1 - q], za[q], twM);
            }
        } else if (ka == 0) {
            // bin H1 q pairs with H1 (C - q); q = 0 is DC with Nyquist; for even C, q = C/2 is
            // bin H/2 (its own mirror)
            cl_dc<C_, KIND>(op, za[0]);
#pragma unroll
            for (int q = 1; 2 * q < C; ++q) cl_pair<C_, KIND>(op, H1 * q, za[q], za[C - q], twM);
            if constexpr (C % 2 == 0) {
                float2 z1 = za[C / 2], z2 = za[C / 2];
                cl_pair<C_, KIND>(op, H / 2, z1, z2, twM);
                za[C / 2] = z2;
            }
        } else {
            // ka = H1/2: bin H1/2 + H1 q pairs with H1/2 + H1 (C - 1 - q); for odd C,
            // q = (C - 1)/2 is bin H/2 (its own mirror)
#pragma unroll
            for (int q = 0; 2 * q + 1 < C; ++q) cl_pair<C_, KIND>(op, ka + H1 * q, za[q], za[C - 1 - q], twM);
            if constexpr (C % 2 == 1) {
                float2 z1 = za[C / 2], z2 = za[C / 2];
                cl_pair<C_, KIND>(op, H / 2, z1, z2, twM);
                za[C / 2] = z2;
            }
        }
        if constexpr (KIND != CL_SPEC) {
            dftR<C, true>(za);
            cl_twiddle<C, true>(za, wa);
#pragma unroll
            for (int q = 0; q < C; ++q) cl_st(cl_map(aa, q), za[q]);
            if (!self) {
                dftR<C, true>(zb);
                cl_twiddle<C, true>(zb, wb);
#pragma unroll
                for (int q = 0; q < C; ++q) cl_st(cl_map(ab, q), zb[q]);
            }
        }
    }
}

// Decimated point access of CTA r: its local point m is the global packed point C m + r.
template <int C, class P>
struct ClDecim {
    P p;
    int rank;
    static constexpr bool kSmem = false;
    // local points that can be nonzero, for a reader that knows its global count
    template <class Q = P>
    __device__ __forceinline__ auto nz() const -> decltype(std::declval<const Q&>().nz()) {
        const int t = p.nz() - rank;
        return t <= 0 ? 0 : (t + C - 1) / C;
    }
    __device__ __forceinline__ float2 operator()(int m) const { return p(m * C + rank); }
    __device__ __forceinline__ void operator()(int m, float2 v) const { p(m * C + rank, v); }
};

// Spectrum (CL_SPEC), correlation sweep (CL_CORR) and one-buffer elementary reconstruction
// (CL_ELEM) on clusters; grid (C x columns, jobs), one cluster per column.
template <int C, int KIND>
__global__ void __launch_bounds__(ClShape<C>::BLOCK, ClShape<C>::MINB) k_cl_col(const ssa_col_job* __restrict__ jobs,
                                                                                  const ssa_tile* __restrict__ tiles,
                                                                                  int ntiles) {
    using S = ClShape<C>;
    extern __shared__ float2 smem[];
    __shared__ double red[32];
    __shared__ double cl_part[S::C];
    float2* s = smem;
    float2* tw1 = s + spad_size(S::H1);
    float2* twM = tw1 + TwSplit<S::LOGH1 + 1>::N;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    // one cluster per column, or per tile of a column list (a persistent form, the resident
    // clusters looping over the list, measured 44% slower per launch: 10.5 vs 7.3 ms)
    int jb, c;
    if (!sweep_column(tiles, ntiles, blockIdx.x / S::C, jb, c)) return;
    const ssa_col_job J = jobs[jb];
    if (c >= J.ncols) return;  // the whole cluster shares c
    load_twiddles<S::LOGH1 + 1>(tw1);
    cl_load_twM<C>(twM);
    // the first pass of the local transform reads the decimated column from global memory
    const ColPts in = KIND == CL_ELEM ? ColPts{J.in2 + (long long)c * J.ld_in2, nullptr, 1.0f, J.n_in2, 0, 0}
                                      : col_pts(J, c);
    fft_block_io<S::LOGH1, false>(s, ClDecim<S::C, ColPts>{in, rank}, SmemPts{s}, tw1);
    cl.sync();
    ClOp op;
    op.X = reinterpret_cast<const float2*>(J.X);
    op.spec = KIND == CL_SPEC ? reinterpret_cast<float2*>(J.spec + (long long)c * J.ld_spec) : nullptr;
    op.us = KIND == CL_ELEM ? reinterpret_cast<const float2*>(J.spec + (long long)c * J.ld_spec) : nullptr;
    op.R = nullptr;
    cl_exchange<C, KIND>((uint32_t)__cvta_generic_to_shared(s), twM, rank, op);
    cl.sync();
    if constexpr (KIND == CL_SPEC) return;
    const float inv_h = 1.0f / (float)S::H;
    if constexpr (KIND == CL_CORR) {
        // the last pass of the local inverse transform writes the decimated output column
        const RealOut out{J.out + (long long)c * J.ld_out, J.n_out, inv_h};
        fft_block_io<S::LOGH1, true>(s, SmemPts{s}, ClDecim<S::C, RealOut>{out, rank}, tw1);
    } else {
        fft_block<S::LOGH1, true>(s, tw1);
        const float sc = J.scale ? (float)J.scale[c] : 1.0f;
        const float* u = J.in + (long long)c * J.ld_in;
        const float* vv = J.in2 + (long long)c * J.ld_in2;
        float* out = J.out + (long long)c * J.ld_out;
        double acc = 0.0;
        for (int m = threadIdx.x; m < S::H1; m += blockDim.x) {
            const float2 z = s[spad(m)];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int t = 2 * (m * S::C + rank) + h;
                if (t >= J.N) continue;
                double p = (double)((h ? z.y : z.x) * inv_h);
                if (edge_diag(t, J.N)) p = (double)sc * diag_sum(u, vv, t, J.n_in, J.n_in2);
                const int cnt = diag_count(t, J.N, J.L, J.K);
                out[t] = (float)(p / (double)cnt);
                acc += p * p / (double)cnt;
            }
        }
        acc = block_sum<double>(acc, red);
        if (threadIdx.x == 0) cl.map_shared_rank(cl_part, 0)[rank] = acc;
        cl.sync();
        if (rank == 0 && threadIdx.x == 0 && J.norm2) {
            double t = 0.0;
            for (int q = 0; q < S::C; ++q) t += cl_part[q];
            J.norm2[c] = t;
        }
    }
}

// Grouped reconstruction from cached spectra on clusters; grid (C, jobs).
template <int C>
__global__ void __launch_bounds__(ClShape<C>::BLOCK, ClShape<C>::MINB) k_cl_recon(const ssa_recon_job* __restrict__ jobs) {
    using S = ClShape<C>;
    extern __shared__ float2 smem[];
    float2* s = smem;
    float2* tw1 = s + spad_size(S::H1);
    float2* twM = tw1 + TwSplit<S::LOGH1 + 1>::N;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const ssa_recon_job J = jobs[blockIdx.y];
    load_twiddles<S::LOGH1 + 1>(tw1);
    cl_load_twM<C>(twM);
    __syncthreads();
    cl.sync();  // every CTA of the cluster is resident before the remote stores
    ClOp op;
    op.X = nullptr;
    op.spec = nullptr;
    op.us = nullptr;
    op.R = &J;
    cl_exchange<C, CL_RECON>((uint32_t)__cvta_generic_to_shared(s), twM, rank, op);
    cl.sync();
    fft_block<S::LOGH1, true>(s, tw1);
    const float inv_h = 1.0f / (float)S::H;
    for (int m = threadIdx.x; m < S::H1; m += blockDim.x) {
        const float2 z = s[spad(m)];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int t = 2 * (m * S::C + rank) + h;
            if (t >= J.N) continue;
            double p = (double)((h ? z.y : z.x) * inv_h);
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
}

template <int C, int KIND>
static int launch_cl_col(const ssa_col_job* jobs, int njobs, int maxcols, cudaStream_t st, const ssa_tile* tiles) {
    using S = ClShape<C>;
    const int sm = cl_smem_f2<C>() * (int)sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(k_cl_col<C, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return (int)e;
    cudaLaunchConfig_t cfg = {};
    // with a column list, njobs is its tile count: one cluster per listed column
    cfg.gridDim = tiles ? dim3(S::C * njobs, 1, 1) : dim3(S::C * maxcols, njobs, 1);
    cfg.blockDim = dim3(S::BLOCK, 1, 1);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = S::C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_cl_col<C, KIND>, jobs, tiles, njobs);
    return launched(e != cudaSuccess ? e : cudaGetLastError());
}

template <int C>
static int launch_cl_recon(const ssa_recon_job* jobs, int njobs, cudaStream_t st) {
    using S = ClShape<C>;
    const int sm = cl_smem_f2<C>() * (int)sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(k_cl_recon<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return (int)e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(S::C, njobs, 1);
    cfg.blockDim = dim3(S::BLOCK, 1, 1);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = S::C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_cl_recon<C>, jobs);
    return launched(e != cudaSuccess ? e : cudaGetLastError());
}

// CTAs per cluster of a size code: 14 -> 2 (when the 2-CTA form of that length is selected),
// 15 -> 4, 16 -> 8, SSA_FFT_3x13 -> 3, SSA_FFT_3x14 -> 6, SSA_FFT_5x13 -> 5.
static int cl_ctas(int code) {
    return code == 14 ? 2 : code == 15 ? 4 : code == 16 ? 8 : code == SSA_FFT_3x13 ? 3 : code == SSA_FFT_3x14 ? 6
         : code == SSA_FFT_5x13 ? 5 : 0;
}

static int cl_col_dispatch(int kind, const ssa_col_job* jobs, int njobs, int maxcols, int code, cudaStream_t st,
                           const ssa_tile* tiles = nullptr) {
#define SSA_CL_CASE(C)                                                                          \
    if (cl_ctas(code) == C) {                                                                   \
        if (kind == CL_SPEC) return launch_cl_col<C, CL_SPEC>(jobs, njobs, maxcols, st, tiles); \
        if (kind == CL_CORR) return launch_cl_col<C, CL_CORR>(jobs, njobs, maxcols, st, tiles); \
        return launch_cl_col<C, CL_ELEM>(jobs, njobs, maxcols, st, tiles);                      \
    }
    SSA_CL_CASE(2)
    SSA_CL_CASE(3)
    SSA_CL_CASE(4)
    SSA_CL_CASE(5)
    SSA_CL_CASE(6)
    SSA_CL_CASE(8)
#undef SSA_CL_CASE
    return (int)cudaErrorInvalidValue;
}

// grouped reconstruction (single-series contexts): power-of-two lengths only
static int cl_recon_dispatch(const ssa_recon_job* jobs, int njobs, int logh, cudaStream_t st) {
    if (logh == 15) return launch_cl_recon<4>(jobs, njobs, st);
    if (logh == 16) return launch_cl_recon<8>(jobs, njobs, st);
    return (int)cudaErrorInvalidValue;
}
