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

// ---------------------------------------------------------------------------------------------
// Row products on the tensor cores: C = A Bm (or sub - A Bm) for A (m x n, column-major, n <= 64)
// and a small Bm (n x p, p <= 64), the operation of k_rowmul.
//
// Both operands are split into three TF32 parts, x = x1 + x2 + x3, by truncation (x1 = x with its
// low 13 mantissa bits cleared, x2 the same of x - x1, x3 = x - x1 - x2: exact for FP32 values,
// ~33 significant bits of an FP64 Bm), and the product is the sum of the six part products down
// to relative size 2^-22: a1 b1 + a1 b2 + a2 b1 + a1 b3 + a2 b2 + a3 b1 (the dropped ones are
// ~2^-33), accumulated in FP32 in TMEM: the rounding of an FP32 product with FP32 accumulation,
// on the tensor pipe.
//   k_split_b (one CTA per job) writes Bm's three parts once, as the shared-memory image of the
//   B operand (N = 64 output columns x K, canonical K-major layout of 8-row x 16-byte core
//   matrices, no swizzle), per phase of 32 inner elements, into the job's Bsplit buffer.
//   k_rowmul_tc: CTAs of 256 threads, each over several 128-row tiles of one job (tile t of the
//   job at blockIdx.x + i gridDim.x; 128 = SSA_ROWMUL_ROWS, so the column-sum partials have the
//   layout of k_rowmul). The B image is copied in once; TMEM (64 columns) is allocated once. Per
//   phase of 32 inner elements two threads per row split 16 values each and store the three A
//   parts (K-major core matrices); one elected thread issues 6 x 4 tcgen05.mma.kind::tf32
//   (M = 128, N = 64, K = 8) and commits them to an mbarrier, and the threads load the next
//   phase's (or the next tile's) values while the MMAs run. Epilogue per tile: tcgen05.ld of
//   the accumulators (warp w: TMEM lanes 32 (w % 4).., columns 32 (w / 4)..) into shared memory
//   as a [column][row] tile, then a warp per column stores 128 consecutive rows (16 bytes per
//   lane) and reduces the column's partial sum.
// Every mbarrier wait is bounded; on a timeout the CTA stops issuing, waits (bounded) for its
// own MMAs, frees its TMEM, records the failure in the self-check word and writes nothing more.
#define RT_THREADS 256
#define RT_KH 32                                 // inner elements per phase
#define RT_TPC 4                                 // row tiles per CTA
#define RT_A_PART (RT_KH / 4 * TC_A_LBO)         // 16 KB: 128 rows x 32 TF32
#define RT_B_PART (RT_KH / 4 * TC_B_LBO)         // 8 KB: 64 columns x 32 TF32
#define RT_B_PHASE (3 * RT_B_PART)               // one phase's B image: 24 KB
#define RT_SMEM (3 * RT_A_PART + 2 * RT_B_PHASE) // 96 KB

__device__ __forceinline__ float rt_trunc(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// x = a + b + c exactly (FP32 input): every subtraction is exact, c has at most 2 significant bits
__device__ __forceinline__ void rt_split3f(float x, float& a, float& b, float& c) {
    a = rt_trunc(x);
    const float r = x - a;
    b = rt_trunc(r);
    c = r - b;
}

__device__ __forceinline__ void rt_split3d(double x, float& a, float& b, float& c) {
    a = rt_trunc((float)x);
    const double r1 = x - (double)a;
    b = rt_trunc((float)r1);
    c = rt_trunc((float)(r1 - (double)b));
}

__global__ void __launch_bounds__(256) k_split_b(const ssa_rowmul_job* __restrict__ jobs) {
    const ssa_rowmul_job J = jobs[blockIdx.x];
    const int n = J.n, p = J.p;
    if (!J.Bsplit || n < 1 || p < 1 || n > SSA_MAX_KP || p > SSA_MAX_KP) return;
    const int nph = (n + RT_KH - 1) / RT_KH;
    unsigned char* img = reinterpret_cast<unsigned char*>(J.Bsplit);
    // element (output column j, inner k): phase k / 32, 4 consecutive k per 16-byte slot
    for (int e = threadIdx.x; e < nph * SSA_MAX_KP * (RT_KH / 4); e += blockDim.x) {
        const int ph = e / (SSA_MAX_KP * (RT_KH / 4));
        const int rem = e - ph * SSA_MAX_KP * (RT_KH / 4);
        const int j = rem % SSA_MAX_KP, s4 = rem / SSA_MAX_KP;
        float b1[4], b2[4], b3[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = ph * RT_KH + 4 * s4 + u;
            double b = 0.0;
            if (j < p && k < n) b = J.Bm64 ? J.Bm64[k + (long long)j * J.ldb] : (double)J.Bm[k + (long long)j * J.ldb];
            rt_split3d(b, b1[u], b2[u], b3[u]);
        }
        unsigned char* base = img + (size_t)ph * RT_B_PHASE + tc_off<TcTF32>(j, 4 * s4, TC_B_LBO);
        *reinterpret_cast<float4*>(base) = make_float4(b1[0], b1[1], b1[2], b1[3]);
        *reinterpret_cast<float4*>(base + RT_B_PART) = make_float4(b2[0], b2[1], b2[2], b2[3]);
        *reinterpret_cast<float4*>(base + 2 * RT_B_PART) = make_float4(b3[0], b3[1], b3[2], b3[3]);
    }
}

__global__ void __launch_bounds__(RT_THREADS) k_rowmul_tc(const ssa_rowmul_job* __restrict__ jobs) {
    extern __shared__ __align__(1024) unsigned char rts[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const ssa_rowmul_job J = jobs[blockIdx.y];
    const int n = J.n, p = J.p;
    const int ntiles = (J.m + SSA_ROWMUL_ROWS - 1) / SSA_ROWMUL_ROWS;
    if ((int)blockIdx.x >= ntiles || !J.Bsplit || n < 1 || p < 1 || n > SSA_MAX_KP || p > SSA_MAX_KP) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char* sA = rts;                  // parts a1, a2, a3 of the phase (the epilogue tile too)
    unsigned char* sB = rts + 3 * RT_A_PART;  // parts b1, b2, b3 of every phase
    const int nph = (n + RT_KH - 1) / RT_KH;

    if (tid == 0) {
        tc_mbar_init(&bar, 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(&tmem_base)),
                     "r"(64)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    {
        const uint4* src = reinterpret_cast<const uint4*>(J.Bsplit);
        uint4* dst = reinterpret_cast<uint4*>(sB);
        for (int u = tid; u < nph * (RT_B_PHASE / 16); u += RT_THREADS) dst[u] = src[u];
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = tc_idesc<TcTF32::FMT>();

    const int r = tid & (SSA_ROWMUL_ROWS - 1), half = tid >> 7;  // row in the tile, inner half
    constexpr int QH = RT_KH / 2;
    float v[QH];
    auto load_a = [&](int t, int ph) {
        const int row = t * SSA_ROWMUL_ROWS + r;
        const bool rok = row < J.m;
        const float* arow = J.A + (long long)row;
#pragma unroll
        for (int q = 0; q < QH; ++q) {
            const int c = ph * RT_KH + half * QH + q;
            v[q] = (rok && c < n) ? arow[(long long)c * J.lda] : 0.f;
        }
    };
    bool ok = true;
    int ncommit = 0;  // commits issued; the mbarrier phase of commit c has parity c & 1
    auto wait_last = [&]() {
        if (ncommit > 0 && ok && !tc_mbar_wait(&bar, (uint32_t)((ncommit - 1) & 1))) ok = false;
    };
    constexpr int CT_LD = SSA_ROWMUL_ROWS + 4;
    float* ct = reinterpret_cast<float*>(rts);  // 64 x CT_LD floats (33.8 KB) over the A stages
    const int sub4 = warp & 3, chalf = warp >> 2;
    const int rl = 4 * lane;
    load_a(blockIdx.x, 0);
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int r0 = t * SSA_ROWMUL_ROWS;
        const int rows = min(SSA_ROWMUL_ROWS, J.m - r0);
        for (int ph = 0; ph < nph; ++ph) {
            wait_last();  // the A stages are free again
#pragma unroll
            for (int s4 = 0; s4 < QH / 4; ++s4) {
                float4 a1, a2, a3;
                rt_split3f(v[4 * s4 + 0], a1.x, a2.x, a3.x);
                rt_split3f(v[4 * s4 + 1], a1.y, a2.y, a3.y);
                rt_split3f(v[4 * s4 + 2], a1.z, a2.z, a3.z);
                rt_split3f(v[4 * s4 + 3], a1.w, a2.w, a3.w);
                const uint32_t off = tc_off<TcTF32>(r, half * QH + 4 * s4, TC_A_LBO);
                *reinterpret_cast<float4*>(sA + off) = a1;
                *reinterpret_cast<float4*>(sA + RT_A_PART + off) = a2;
                *reinterpret_cast<float4*>(sA + 2 * RT_A_PART + off) = a3;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_fence_before();
            if (!ok) failed = 1;
            __syncthreads();
            if (tid == 0 && !failed) {
                tc_fence_after();
                const uint32_t a0 = tc_smem_u32(sA), b0 = tc_smem_u32(sB) + (uint32_t)(ph * RT_B_PHASE);
                const int live = min(RT_KH, n - ph * RT_KH);
                const int nks = (live + TcTF32::MMA_K - 1) / TcTF32::MMA_K;
                // part products (A part, B part), largest first
                auto product = [&](int ia, int ib, bool first) {
                    for (int ks = 0; ks < nks; ++ks) {
                        const uint64_t da = tc_desc(a0 + ia * RT_A_PART + ks * 2 * TC_A_LBO, TC_A_LBO, 128);
                        const uint64_t db = tc_desc(b0 + ib * RT_B_PART + ks * 2 * TC_B_LBO, TC_B_LBO, 128);
                        tc_mma<TcTF32>(tmem, da, db, idesc, (!first || ks > 0) ? 1u : 0u);
                    }
                };
                product(0, 0, ph == 0);
                product(0, 1, false);
                product(1, 0, false);
                product(0, 2, false);
                product(1, 1, false);
                product(2, 0, false);
                tc_commit(&bar);
            }
            if (failed) break;
            ++ncommit;
            // the next phase's values, or the next tile's first, in flight while the MMAs run
            if (ph + 1 < nph) load_a(t, ph + 1);
            else if (t + (int)gridDim.x < ntiles) load_a(t + gridDim.x, 0);
        }
        if (failed) break;
        wait_last();  // the tile's MMAs are done: TMEM and the A stages may be read
        if (!ok) failed = 1;
        __syncthreads();
        if (failed) break;
        tc_fence_after();
        {
            const uint32_t lane_base = (uint32_t)(sub4 * 32) << 16;
            const int rr = sub4 * 32 + lane;
            for (int cb = chalf * 32; cb < min(p, chalf * 32 + 32); cb += 8) {
                float x[8];
                tc_ld8(tmem + lane_base + (uint32_t)cb, x);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int q = 0; q < 8; ++q) ct[(cb + q) * CT_LD + rr] = x[q];
            }
        }
        tc_fence_before();  // the accumulator reads are complete before the next tile's MMAs
        __syncthreads();
        const bool vecC = rl + 4 <= rows && ((reinterpret_cast<uintptr_t>(J.C) & 15) == 0) && ((J.ldc & 3) == 0) &&
                          (!J.sub || (((reinterpret_cast<uintptr_t>(J.sub) & 15) == 0) && ((J.ldsub & 3) == 0)));
        for (int col = warp; col < p; col += RT_THREADS / 32) {
            float4 y = *reinterpret_cast<const float4*>(ct + col * CT_LD + rl);
            const long long cbase = (long long)(r0 + rl) + (long long)col * J.ldc;
            double cs = 0.0;
            if (vecC) {
                if (J.sub) {
                    const float4 sv =
                        *reinterpret_cast<const float4*>(J.sub + (long long)(r0 + rl) + (long long)col * J.ldsub);
                    y = make_float4(sv.x - y.x, sv.y - y.y, sv.z - y.z, sv.w - y.w);
                }
                *reinterpret_cast<float4*>(J.C + cbase) = y;
                cs = (double)y.x + (double)y.y + (double)y.z + (double)y.w;
            } else {
                float yv[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (rl + u < rows) {
                        if (J.sub) yv[u] = J.sub[(long long)(r0 + rl + u) + (long long)col * J.ldsub] - yv[u];
                        J.C[cbase + u] = yv[u];
                        cs += (double)yv[u];
                    }
            }
            if (J.colsum) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) cs += __shfl_xor_sync(0xffffffffu, cs, o);
                if (lane == 0) J.colsum[(long long)t * p + col] = cs;
            }
        }
        __syncthreads();  // every warp is done with the tile before the next tile's A parts overwrite it
    }
    if (failed) {
        tc_mbar_wait(&bar, (uint32_t)((ncommit - 1) & 1));  // bounded: own MMAs done
        if (tid == 0) check_fail(10, 1, (unsigned)blockIdx.x);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
}

static int launch_rowmul_tc(const ssa_rowmul_job* jobs, int njobs, int maxrows, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(k_rowmul_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, RT_SMEM);
    if (e != cudaSuccess) return (int)e;
    k_split_b<<<njobs, 256, 0, st>>>(jobs);
    if ((e = cudaGetLastError()) != cudaSuccess) return launched(e);
    launched(e);
    const int tiles = (maxrows + SSA_ROWMUL_ROWS - 1) / SSA_ROWMUL_ROWS;
    k_rowmul_tc<<<dim3((tiles + RT_TPC - 1) / RT_TPC, njobs), RT_THREADS, RT_SMEM, st>>>(jobs);
    return launched(cudaGetLastError());
}
