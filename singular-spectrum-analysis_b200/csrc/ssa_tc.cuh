// W-correlation Gram on the 5th-generation tensor cores (tcgen05, accumulators in TMEM).
//
// G = X diag(w) X^T for the k <= 64 elementary reconstructions X (k x N, component rows
// contiguous in time) of one series, w_t = diagonal count. Each CTA (128 threads) owns one
// (series, time chunk) and forms its chunk's partial Gram:
//   - time tiles of 32 steps: X scaled by sqrt(w_t) is split in registers into two parts of the
//     operand type, hi = round(x), lo = round(x - hi) (TF32: 11 significant bits each, the pair
//     ~22 bits; BF16: 8 bits each, the pair ~16 bits), written to shared memory in the canonical
//     K-major layout without swizzle (8-row x 16-byte core matrices; LBO = next 16 bytes of K,
//     SBO = next 8 rows);
//   - A = [hi; lo] (M = 128 rows) and B = hi (N = 64 rows): one tcgen05.mma (kind::tf32 per 8
//     time steps, or kind::f16 with BF16 operands per 16) accumulates both hi hi^T and lo hi^T
//     in FP32 in TMEM (128 lanes x 64 columns);
//   - two operand stages; one elected thread issues the MMAs and commits them to the stage's
//     mbarrier, which the writers wait on before refilling the stage;
//   - epilogue: tcgen05.ld of the accumulator, G_ij = HH_ij + LH_ij + LH_ji in FP64 (lo lo^T, of
//     relative size 2^-22 for TF32, 2^-16 for BF16, is dropped), packed upper triangle into the
//     chunk's partial slot (the layout k_gram writes, so k_wfin reduces either).
// k_gram_f32 below is the same chunked Gram with FP32 products and FP32 accumulation on the
// CUDA cores, for comparison.
// Every wait on an mbarrier is bounded; a wait that runs out records an error in the job's
// status word and the kernel leaves after waiting (bounded) for its own MMAs, freeing TMEM.

#include <cuda_bf16.h>

#define TC_THREADS 128
#define TC_KT 32                                   // time steps per tile (K)
#define TC_M 128                                   // A rows: 64 hi + 64 lo
#define TC_N 64                                    // B rows (components)
#define TC_A_LBO (TC_M / 8 * 128)                  // bytes between 16-byte K slices of A
#define TC_B_LBO (TC_N / 8 * 128)
#define TC_EPI_LD (TC_N + 1)
#define TC_EPI_BYTES (TC_M * TC_EPI_LD * 4)        // epilogue staging over the idle stages
#define TC_WAIT_LIMIT (1 << 22)

// Operand precisions of the split products: element bytes, elements per 16-byte K slice, K per
// instruction, the instruction descriptor's A / B format code (kind::tf32: 2; kind::f16: 1 =
// BF16).
struct TcTF32 {
    static constexpr int BYTES = 4, EPS = 4, MMA_K = 8, FMT = 2;
};
struct TcBF16 {
    static constexpr int BYTES = 2, EPS = 8, MMA_K = 16, FMT = 1;
};
template <class P>
struct TcShape {
    static constexpr int A_BYTES = TC_KT / P::EPS * TC_A_LBO;  // TF32 16 KB, BF16 8 KB
    static constexpr int B_BYTES = TC_KT / P::EPS * TC_B_LBO;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr int SMEM = 2 * STAGE > TC_EPI_BYTES ? 2 * STAGE : TC_EPI_BYTES;
};

__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor: K-major, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor: D f32, A and B of format FMT (both the same type), both K-major,
// N = 64, M = 128.
template <int FMT>
__device__ __forceinline__ uint32_t tc_idesc() {
    return (1u << 4) | ((uint32_t)FMT << 7) | ((uint32_t)FMT << 10) | ((uint32_t)(TC_N >> 3) << 17) |
           ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ float tc_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__device__ __forceinline__ void tc_mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(bar)), "r"(count) : "memory");
}

// Bounded wait for completion of the phase with the given parity; false when the limit ran out.
__device__ __forceinline__ bool tc_mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = tc_smem_u32(bar);
    for (int it = 0; it < TC_WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <class P>
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accum) {
    if constexpr (P::FMT == 2)
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
            :
            : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accum)
            : "memory");
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            :
            : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accum)
            : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tc_smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_ld8(uint32_t taddr, float* v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row r, time j) of a K-major tile whose 16-byte K slices (P::EPS
// elements) are lbo bytes apart.
template <class P>
__device__ __forceinline__ uint32_t tc_off(int r, int j, uint32_t lbo) {
    return (uint32_t)(j / P::EPS) * lbo + (uint32_t)(r >> 3) * 128u + (uint32_t)(r & 7) * 16u +
           (uint32_t)(j % P::EPS) * (uint32_t)P::BYTES;
}

__device__ __forceinline__ uint32_t tc_bf16x2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a in the low half
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Split four consecutive time values of row c into hi / lo parts and store them: hi at A row c
// and B row c, lo at A row c + 64 (TF32: one 16-byte slice each).
__device__ __forceinline__ void tc_store4(const float* x, unsigned char* sA, unsigned char* sB, int c, int j) {
    float4 h, l;
    h.x = tc_tf32(x[0]);
    h.y = tc_tf32(x[1]);
    h.z = tc_tf32(x[2]);
    h.w = tc_tf32(x[3]);
    l.x = x[0] - h.x;
    l.y = x[1] - h.y;
    l.z = x[2] - h.z;
    l.w = x[3] - h.w;
    *reinterpret_cast<float4*>(sA + tc_off<TcTF32>(c, j, TC_A_LBO)) = h;
    *reinterpret_cast<float4*>(sA + tc_off<TcTF32>(c + 64, j, TC_A_LBO)) = l;
    *reinterpret_cast<float4*>(sB + tc_off<TcTF32>(c, j, TC_B_LBO)) = h;
}

// The same for eight consecutive values as BF16 (one 16-byte slice each).
__device__ __forceinline__ void tc_store8_bf16(const float* x, unsigned char* sA, unsigned char* sB, int c, int j) {
    uint32_t hw[4], lw[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(x[2 * q], x[2 * q + 1]);
        const float2 hf = __bfloat1622float2(h);
        hw[q] = *reinterpret_cast<const uint32_t*>(&h);
        lw[q] = tc_bf16x2(x[2 * q] - hf.x, x[2 * q + 1] - hf.y);
    }
    const uint4 hv = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    const uint4 lv = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    *reinterpret_cast<uint4*>(sA + tc_off<TcBF16>(c, j, TC_A_LBO)) = hv;
    *reinterpret_cast<uint4*>(sA + tc_off<TcBF16>(c + 64, j, TC_A_LBO)) = lv;
    *reinterpret_cast<uint4*>(sB + tc_off<TcBF16>(c, j, TC_B_LBO)) = hv;
}

template <class P>
__global__ void __launch_bounds__(TC_THREADS) k_gram_tc(const ssa_wgram_job* __restrict__ jobs) {
    using S = TcShape<P>;
    extern __shared__ __align__(1024) unsigned char tsm[];
    __shared__ __align__(8) uint64_t bar[3];
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const ssa_gram_job J = jobs[blockIdx.y].g;
    int* const status = jobs[blockIdx.y].status;
    const int chunk = blockIdx.x;
    const int t_begin = chunk * J.rows_per_cta;
    if (t_begin >= J.m) return;
    const int t_end = min(J.m, t_begin + J.rows_per_cta);
    const int n = J.n;
    const int tid = threadIdx.x, warp = tid >> 5;

    if (tid == 0) {
        tc_mbar_init(&bar[0], 1);
        tc_mbar_init(&bar[1], 1);
        tc_mbar_init(&bar[2], 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(&tmem_base)),
                     "r"(64)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = tc_idesc<P::FMT>();

    // each thread fills 16 consecutive time steps of one component row per tile; the next tile's
    // values are loaded while the tensor cores work on the current one
    const int c = tid >> 1;
    const int j0 = (tid & 1) * 16;
    const float* xrow = J.A + (long long)c * J.ld;
    const int ntiles = (t_end - t_begin + TC_KT - 1) / TC_KT;
    float v[16];
    auto load_tile = [&](int it) {
        const int t0 = t_begin + it * TC_KT + j0;
        if (c < n && t0 + 16 <= t_end) {
            const float4* p4 = reinterpret_cast<const float4*>(xrow + t0);  // 16-byte aligned
#pragma unroll
            for (int q4 = 0; q4 < 4; ++q4) {
                const float4 a = p4[q4];
                v[4 * q4 + 0] = a.x;
                v[4 * q4 + 1] = a.y;
                v[4 * q4 + 2] = a.z;
                v[4 * q4 + 3] = a.w;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = (c < n && t0 + q < t_end) ? xrow[t0 + q] : 0.f;
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int t = min(t0 + q, J.N - 1);
            v[q] *= sqrtf((float)diag_count(t, J.N, J.L, J.K));
        }
    };
    bool ok = true;
    if (ntiles > 0) load_tile(0);
    for (int it = 0; it < ntiles; ++it) {
        const int stage = it & 1;
        unsigned char* sA = tsm + stage * S::STAGE;
        unsigned char* sB = sA + S::A_BYTES;
        if (it >= 2 && !tc_mbar_wait(&bar[stage], ((it >> 1) - 1) & 1)) ok = false;
        if constexpr (P::FMT == 2) {
#pragma unroll
            for (int q4 = 0; q4 < 4; ++q4) tc_store4(v + 4 * q4, sA, sB, c, j0 + 4 * q4);
        } else {
#pragma unroll
            for (int q8 = 0; q8 < 2; ++q8) tc_store8_bf16(v + 8 * q8, sA, sB, c, j0 + 8 * q8);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = tc_smem_u32(sA), b0 = tc_smem_u32(sB);
            // one instruction covers MMA_K elements = 32 bytes of K = two slices
#pragma unroll
            for (int ks = 0; ks < TC_KT / P::MMA_K; ++ks) {
                const uint64_t da = tc_desc(a0 + ks * 2 * TC_A_LBO, TC_A_LBO, 128);
                const uint64_t db = tc_desc(b0 + ks * 2 * TC_B_LBO, TC_B_LBO, 128);
                tc_mma<P>(tmem, da, db, idesc, (it > 0 || ks > 0) ? 1u : 0u);
            }
            tc_commit(&bar[stage]);
        }
        if (it + 1 < ntiles) load_tile(it + 1);
    }
    // the last tile's commit completes after every earlier MMA
    if (ntiles > 0 && !tc_mbar_wait(&bar[(ntiles - 1) & 1], ((ntiles - 1) >> 1) & 1)) ok = false;
    if (!ok) failed = 1;
    __syncthreads();
    if (failed && ntiles > 0) tc_mbar_wait(&bar[(ntiles - 1) & 1], ((ntiles - 1) >> 1) & 1);  // bounded
    __syncthreads();
    tc_fence_after();
    float* epi = reinterpret_cast<float*>(tsm);  // 128 x TC_EPI_LD floats, over the idle stages
    if (!failed && ntiles > 0) {
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
#pragma unroll
        for (int cb = 0; cb < TC_N; cb += 8) {
            float v[8];
            tc_ld8(tmem + lane_base + (uint32_t)cb, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 8; ++q) epi[tid * TC_EPI_LD + cb + q] = v[q];
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
    if (failed) {
        if (tid == 0 && status) atomicOr(status, 8);
        if (tid == 0) check_fail(9, 1, (unsigned)chunk);
        return;
    }
    double* part = J.part + (long long)chunk * (n * (n + 1) / 2);
    const int np = n * (n + 1) / 2;
    for (int e = tid; e < np; e += TC_THREADS) {
        // e -> (i, j), i <= j, row-major packed upper triangle
        int i = 0, rem = e;
        while (rem >= n - i) {
            rem -= n - i;
            ++i;
        }
        const int j = i + rem;
        double g = 0.0;
        if (ntiles > 0)
            g = (double)epi[i * TC_EPI_LD + j] + (double)epi[(64 + i) * TC_EPI_LD + j] +
                (double)epi[(64 + j) * TC_EPI_LD + i];
        part[pk_index(i, j, n)] = g;
    }
}

// The chunked weighted Gram with FP32 products and FP32 accumulation on the CUDA cores: one CTA
// of 256 threads per (chunk, job); time tiles of 32 steps scaled by sqrt(w_t) staged in shared
// memory ([time][component], padded), thread (ty, tx) of a 16 x 16 grid accumulating the 4 x 4
// block of G at rows 4 ty.., columns 4 tx..; FP64 partials in the packed layout of k_gram.
#define GF_THREADS 256
#define GF_LD (TC_N + 4)
__global__ void __launch_bounds__(GF_THREADS) k_gram_f32(const ssa_wgram_job* __restrict__ jobs) {
    __shared__ __align__(16) float tile[TC_KT * GF_LD];
    const ssa_gram_job J = jobs[blockIdx.y].g;
    const int t_begin = blockIdx.x * J.rows_per_cta;
    if (t_begin >= J.m) return;
    const int t_end = min(J.m, t_begin + J.rows_per_cta);
    const int n = J.n;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
    const bool live = 4 * ty < n && 4 * tx < n && ty <= tx;  // blocks on or above the diagonal
    for (int t0 = t_begin; t0 < t_end; t0 += TC_KT) {
        __syncthreads();
        for (int e = threadIdx.x; e < TC_KT * TC_N; e += GF_THREADS) {
            const int c = e / TC_KT, j = e - c * TC_KT;  // time fastest: coalesced row reads
            const int t = t0 + j;
            float v = 0.f;
            if (c < n && t < t_end) v = J.A[(long long)c * J.ld + t] * sqrtf((float)diag_count(t, J.N, J.L, J.K));
            tile[j * GF_LD + c] = v;
        }
        __syncthreads();
        if (live) {
#pragma unroll 8
            for (int j = 0; j < TC_KT; ++j) {
                const float4 a = *reinterpret_cast<const float4*>(tile + j * GF_LD + 4 * ty);
                const float4 b = *reinterpret_cast<const float4*>(tile + j * GF_LD + 4 * tx);
                const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
                for (int p = 0; p < 4; ++p)
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[p][q] = fmaf(av[p], bv[q], acc[p][q]);
            }
        }
    }
    if (!live) return;
    double* part = J.part + (long long)blockIdx.x * (n * (n + 1) / 2);
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int i = 4 * ty + p, j = 4 * tx + q;
            if (i < n && j < n && i <= j) part[pk_index(i, j, n)] = (double)acc[p][q];
        }
}

// Launchers: one CTA per (chunk, job); chunks of rows_per_cta time steps (multiple of 32).
template <class P>
static int launch_gram_tc_p(const ssa_wgram_job* jobs, int njobs, int maxchunks, cudaStream_t st) {
    constexpr int smem = TcShape<P>::SMEM;
    cudaError_t e = cudaFuncSetAttribute(k_gram_tc<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return (int)e;
    k_gram_tc<P><<<dim3(maxchunks, njobs), TC_THREADS, smem, st>>>(jobs);
    return launched(cudaGetLastError());
}

// mode: 1 split TF32, 2 split BF16 (tensor cores), 3 FP32 (CUDA cores)
static int launch_gram_tc(const ssa_wgram_job* jobs, int njobs, int maxchunks, int mode, cudaStream_t st) {
    if (mode == 2) return launch_gram_tc_p<TcBF16>(jobs, njobs, maxchunks, st);
    if (mode == 3) {
        k_gram_f32<<<dim3(maxchunks, njobs), GF_THREADS, 0, st>>>(jobs);
        return launched(cudaGetLastError());
    }
    return launch_gram_tc_p<TcTF32>(jobs, njobs, maxchunks, st);
}
