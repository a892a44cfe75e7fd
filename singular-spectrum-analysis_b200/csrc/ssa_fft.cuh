// Shared-memory FFT building blocks for the SSA hot path on sm_100a.
//
// One CTA transforms one real sequence of length M = 2H (H = 2^LOGH complex points) that is
// packed as z[n] = a[2n] + i a[2n+1]. The complex FFT of length H runs as a Stockham
// auto-sort FFT (Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC'08) with radix-16 (and lane-pair radix-32) passes held in
// registers: every thread owns 16 points per pass, loads them, applies twiddles and the
// in-register DFT, waits at a barrier and stores them at their auto-sorted positions, so the
// transform runs in place in one buffer of H points. The buffer is padded by one point per 16
// (spad) so that both the strided loads and the auto-sort stores of a half-warp touch 16
// distinct 8-byte bank pairs.
//
// Twiddles come from one table g_tw[t] = exp(-2 pi i t / TW_N), computed on the host in FP64
// and rounded to FP32 once per device.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#define SSA_TW_LOG 17
#define SSA_TW_N (1 << SSA_TW_LOG)
// Largest complex FFT a single CTA holds: H = 2^14 points (real length M = 32768).
#define SSA_MAX_LOGH 14
#define SSA_MIN_LOGH 4

// Defined once in the translation unit that includes this header (ssa_kernels.cu).
__device__ float2 g_tw[SSA_TW_N];
// Twiddles of the lengths 3 * 2^A: g_tw3[t] = exp(-2 pi i t / (3 * 2^15)), FP64 on the host.
#define SSA_TW3_LOG 15
#define SSA_TW3_N (3 << SSA_TW3_LOG)
__device__ float2 g_tw3[SSA_TW3_N];
// Twiddles of the length 5 * 2^14: g_tw5[t] = exp(-2 pi i t / (5 * 2^14)), FP64 on the host.
#define SSA_TW5_LOG 14
#define SSA_TW5_N (5 << SSA_TW5_LOG)
__device__ float2 g_tw5[SSA_TW5_N];

namespace ssa {

__device__ __forceinline__ int spad(int a) { return a + (a >> 4); }
__host__ __device__ constexpr int spad_size(int h) { return h + (h >> 4) + 16; }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// Two-level twiddle table in shared memory for resolution M = 2^LOGM:
//   W_M^t = hi[t >> LO] * lo[t & (2^LO - 1)],  lo[j] = W_M^j,  hi[i] = W_M^(i 2^LO).
// Each factor is a correctly rounded FP32 value from the FP64-computed global table, so a
// twiddle costs two shared loads and one complex multiply (~1 ulp extra error).
template <int LOGM>
struct TwSplit {
    static constexpr int LO = (LOGM + 1) / 2;
    static constexpr int HI = LOGM - LO;
    static constexpr int NLO = 1 << LO;
    static constexpr int NHI = 1 << HI;
    static constexpr int N = NLO + NHI;  // float2 entries
};

// Fill the table (lo first, then hi); caller syncs before use.
template <int LOGM>
__device__ __forceinline__ void load_twiddles(float2* tab) {
    using S = TwSplit<LOGM>;
    static_assert(LOGM <= SSA_TW_LOG, "twiddle resolution exceeds the global table");
    for (int i = threadIdx.x; i < S::N; i += blockDim.x) {
        const int t = i < S::NLO ? i : (i - S::NLO) << S::LO;
        tab[i] = g_tw[t << (SSA_TW_LOG - LOGM)];
    }
}

// The same two-level table for the resolutions M = 3 * 2^A (9 <= A <= SSA_TW3_LOG): lo holds
// W_M^j for j < 512, hi W_M^(512 i) for i < M / 512.
template <int A>
struct TwSplit3 {
    static constexpr int LO = 9;
    static constexpr int NLO = 1 << LO;
    static constexpr int NHI = 3 << (A - LO);
    static constexpr int N = NLO + NHI;
};

template <int A>
__device__ __forceinline__ void load_twiddles3(float2* tab) {
    using S = TwSplit3<A>;
    static_assert(A >= S::LO && A <= SSA_TW3_LOG, "twiddle resolution outside the 3 * 2^A table");
    for (int i = threadIdx.x; i < S::N; i += blockDim.x) {
        const int t = i < S::NLO ? i : (i - S::NLO) << S::LO;
        tab[i] = g_tw3[t << (SSA_TW3_LOG - A)];
    }
}

// The same for the resolution M = 5 * 2^14: lo W_M^j for j < 512, hi W_M^(512 i) for i < M / 512.
template <int A>
struct TwSplit5 {
    static constexpr int LO = 9;
    static constexpr int NLO = 1 << LO;
    static constexpr int NHI = 5 << (A - LO);
    static constexpr int N = NLO + NHI;
};

template <int A>
__device__ __forceinline__ void load_twiddles5(float2* tab) {
    using S = TwSplit5<A>;
    static_assert(A >= S::LO && A <= SSA_TW5_LOG, "twiddle resolution outside the 5 * 2^A table");
    for (int i = threadIdx.x; i < S::N; i += blockDim.x) {
        const int t = i < S::NLO ? i : (i - S::NLO) << S::LO;
        tab[i] = g_tw5[t << (SSA_TW5_LOG - A)];
    }
}

// W_M^t (forward sign) or its conjugate from a two-level table with split S, t in [0, M)
template <class S, bool INV>
__device__ __forceinline__ float2 twiddle_s(const float2* tab, int t) {
    float2 w = cmul(tab[S::NLO + (t >> S::LO)], tab[t & (S::NLO - 1)]);
    if (INV) w.y = -w.y;
    return w;
}

// W_M^t (forward sign) or its conjugate, t in [0, M), M = 2^LOGM
template <int LOGM, bool INV>
__device__ __forceinline__ float2 twiddle(const float2* tab, int t) {
    return twiddle_s<TwSplit<LOGM>, INV>(tab, t);
}

// Multiply by the constant W_16^e (forward sign) or its conjugate.
template <bool INV, int E>
__device__ __forceinline__ float2 w16(float2 a) {
    constexpr float C1 = 0.92387953251128674f;  // cos(pi/8)
    constexpr float S1 = 0.38268343236508978f;  // sin(pi/8)
    constexpr float R2 = 0.70710678118654752f;  // 1/sqrt(2)
    constexpr int e = E & 15;
    float2 w = make_float2(1.f, 0.f);
    if constexpr (e == 0) return a;
    else if constexpr (e == 1) w = make_float2(C1, -S1);
    else if constexpr (e == 2) w = make_float2(R2, -R2);
    else if constexpr (e == 3) w = make_float2(S1, -C1);
    else if constexpr (e == 4) return mul_mi<INV>(a);
    else if constexpr (e == 6) w = make_float2(-R2, -R2);
    else if constexpr (e == 9) w = make_float2(-C1, S1);
    else static_assert(e == 0, "unused constant");
    if (INV) w.y = -w.y;
    return cmul(a, w);
}

template <bool INV>
__device__ __forceinline__ void dft2(float2* a) {
    float2 t = a[0];
    a[0] = cadd(t, a[1]);
    a[1] = csub(t, a[1]);
}

template <bool INV>
__device__ __forceinline__ void dft4s(float2& a0, float2& a1, float2& a2, float2& a3) {
    float2 s0 = cadd(a0, a2), d0 = csub(a0, a2);
    float2 s1 = cadd(a1, a3), d1 = mul_mi<INV>(csub(a1, a3));
    a0 = cadd(s0, s1);
    a2 = csub(s0, s1);
    a1 = cadd(d0, d1);
    a3 = csub(d0, d1);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2* a) { dft4s<INV>(a[0], a[1], a[2], a[3]); }

// 8 = 2 x 4: inner DFT4 over a[j + 2l], twiddle W8^{jm} = W16^{2jm}, outer DFT2 over j,
// output index m + 4n.
template <bool INV>
__device__ __forceinline__ void dft8(float2* a) {
    float2 b0[4] = {a[0], a[2], a[4], a[6]};
    float2 b1[4] = {a[1], a[3], a[5], a[7]};
    dft4<INV>(b0);
    dft4<INV>(b1);
    b1[1] = w16<INV, 2>(b1[1]);
    b1[2] = w16<INV, 4>(b1[2]);
    b1[3] = w16<INV, 6>(b1[3]);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        a[m] = cadd(b0[m], b1[m]);
        a[m + 4] = csub(b0[m], b1[m]);
    }
}

// Inner stage of the 16-point DFT below for inputs of which only a[0 .. NZ) may be nonzero
// (NZ = 4, 8 or 16; a[NZ ..] are not read): DFT4 over a[j + 4l] (l) for each j < 4, with the
// terms of the zero inputs left out. Equal to the full stage on such inputs (up to the sign of
// zero results).
template <bool INV, int NZ>
__device__ __forceinline__ void dft16_inner(float2* a) {
    static_assert(NZ == 4 || NZ == 8 || NZ == 16, "inner stage for 4, 8 or 16 nonzero inputs");
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if constexpr (NZ == 16) {
            dft4s<INV>(a[j], a[j + 4], a[j + 8], a[j + 12]);
        } else if constexpr (NZ == 8) {
            const float2 x0 = a[j], x1 = a[j + 4], m1 = mul_mi<INV>(x1);
            a[j] = cadd(x0, x1);
            a[j + 4] = cadd(x0, m1);
            a[j + 8] = csub(x0, x1);
            a[j + 12] = csub(x0, m1);
        } else {
            a[j + 4] = a[j + 8] = a[j + 12] = a[j];
        }
    }
}

// 16 = 4 x 4: inner DFT4 over a[j + 4l] (l), twiddle W16^{jm}, outer DFT4 over j,
// output index m + 4n. With NZ < 16, only a[0 .. NZ) may be nonzero (dft16_inner).
template <bool INV, int NZ = 16>
__device__ __forceinline__ void dft16(float2* a) {
    dft16_inner<INV, NZ>(a);
    // b[j][m] sits at a[j + 4m]
    a[5] = w16<INV, 1>(a[5]);
    a[9] = w16<INV, 2>(a[9]);
    a[13] = w16<INV, 3>(a[13]);
    a[6] = w16<INV, 2>(a[6]);
    a[10] = w16<INV, 4>(a[10]);
    a[14] = w16<INV, 6>(a[14]);
    a[7] = w16<INV, 3>(a[7]);
    a[11] = w16<INV, 6>(a[11]);
    a[15] = w16<INV, 9>(a[15]);
    // outer DFT4 over j for each m: inputs a[4m + j], outputs X[m + 4n]
    dft4s<INV>(a[0], a[1], a[2], a[3]);
    dft4s<INV>(a[4], a[5], a[6], a[7]);
    dft4s<INV>(a[8], a[9], a[10], a[11]);
    dft4s<INV>(a[12], a[13], a[14], a[15]);
    // now a[4m + n] holds X[m + 4n]: transpose 4x4 into natural order
    float2 t;
#define SSA_SWP(i, j) t = a[i]; a[i] = a[j]; a[j] = t;
    SSA_SWP(1, 4) SSA_SWP(2, 8) SSA_SWP(3, 12) SSA_SWP(6, 9) SSA_SWP(7, 13) SSA_SWP(11, 14)
#undef SSA_SWP
}

// 3 points: X1,2 = a0 - (a1 + a2)/2 -/+ i (sqrt 3 / 2)(a1 - a2) (signs of i flipped for INV).
template <bool INV>
__device__ __forceinline__ void dft3(float2* a) {
    constexpr float H3 = 0.86602540378443865f;  // sqrt(3) / 2
    const float2 s = cadd(a[1], a[2]);
    const float2 m = make_float2(a[0].x - 0.5f * s.x, a[0].y - 0.5f * s.y);
    const float2 d = cscale(mul_mi<INV>(csub(a[1], a[2])), H3);
    a[0] = cadd(a[0], s);
    a[1] = cadd(m, d);
    a[2] = csub(m, d);
}

// 6 = 3 x 2: B_r = DFT3 of a[r], a[r + 2], a[r + 4]; X[k] = B_0[k] + W6^k B_1[k],
// X[k + 3] = B_0[k] - W6^k B_1[k], k < 3.
template <bool INV>
__device__ __forceinline__ void dft6(float2* a) {
    constexpr float H3 = 0.86602540378443865f;
    float2 b0[3] = {a[0], a[2], a[4]};
    float2 b1[3] = {a[1], a[3], a[5]};
    dft3<INV>(b0);
    dft3<INV>(b1);
    const float sg = INV ? 1.f : -1.f;
    b1[1] = cmul(b1[1], make_float2(0.5f, sg * H3));
    b1[2] = cmul(b1[2], make_float2(-0.5f, sg * H3));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        a[k] = cadd(b0[k], b1[k]);
        a[k + 3] = csub(b0[k], b1[k]);
    }
}

// 5 points from the definition, pairing n with 5 - n: with s_n = a_n + a_{5-n}, d_n = a_n - a_{5-n},
// X_0 = a_0 + s_1 + s_2, X_{1,4} = a_0 + c_1 s_1 + c_2 s_2 -/+ i (g_1 d_1 + g_2 d_2),
// X_{2,3} = a_0 + c_2 s_1 + c_1 s_2 -/+ i (g_2 d_1 - g_1 d_2), c_j = cos(2 pi j / 5),
// g_j = sin(2 pi j / 5) (signs of i flipped for INV).
template <bool INV>
__device__ __forceinline__ void dft5(float2* a) {
    constexpr float C1 = 0.30901699437494742f, C2 = -0.80901699437494742f;
    constexpr float G1 = 0.95105651629515357f, G2 = 0.58778525229247313f;
    const float2 s1 = cadd(a[1], a[4]), d1 = csub(a[1], a[4]);
    const float2 s2 = cadd(a[2], a[3]), d2 = csub(a[2], a[3]);
    const float2 t1 = make_float2(a[0].x + C1 * s1.x + C2 * s2.x, a[0].y + C1 * s1.y + C2 * s2.y);
    const float2 t2 = make_float2(a[0].x + C2 * s1.x + C1 * s2.x, a[0].y + C2 * s1.y + C1 * s2.y);
    const float2 u1 = mul_mi<INV>(make_float2(G1 * d1.x + G2 * d2.x, G1 * d1.y + G2 * d2.y));
    const float2 u2 = mul_mi<INV>(make_float2(G2 * d1.x - G1 * d2.x, G2 * d1.y - G1 * d2.y));
    a[0] = cadd(a[0], cadd(s1, s2));
    a[1] = cadd(t1, u1);
    a[4] = csub(t1, u1);
    a[2] = cadd(t2, u2);
    a[3] = csub(t2, u2);
}

template <int R, bool INV>
__device__ __forceinline__ void dftR(float2* a) {
    if constexpr (R == 2) dft2<INV>(a);
    else if constexpr (R == 3) dft3<INV>(a);
    else if constexpr (R == 5) dft5<INV>(a);
    else if constexpr (R == 4) dft4<INV>(a);
    else if constexpr (R == 6) dft6<INV>(a);
    else if constexpr (R == 8) dft8<INV>(a);
    else dft16<INV>(a);
}

// Threads that take part in an H-point transform: 16 points each.
template <int LOGH>
struct FftShape {
    static constexpr int H = 1 << LOGH;
    static constexpr int T = H / 16;
    static constexpr int BLOCK = T < 32 ? 32 : T;
    // CTAs per SM the single-buffer kernels are compiled for: 64 registers per thread.
    static constexpr int MINB = 1024 / BLOCK;
};

// Point access of a pass: the padded shared buffer, or (first / last pass only) a functor that
// reads the input point z[i] from global memory / writes the output point z[i] there. A pass
// that reads global memory needs no barrier before its shared stores, and one that writes
// global memory needs none after them; a caller that reuses the buffer after a transform whose
// last pass wrote global memory syncs first.
struct SmemPts {
    float2* s;
    static constexpr bool kSmem = true;
    __device__ __forceinline__ float2 operator()(int i) const { return s[spad(i)]; }
    __device__ __forceinline__ void operator()(int i, float2 v) const { s[spad(i)] = v; }
};

// Point readers that know how many leading points can be nonzero (nz()): the first pass skips
// the rest.
template <class P, class = void>
struct HasNz {
    static constexpr bool value = false;
};
template <class P>
struct HasNz<P, decltype((void)std::declval<const P&>().nz())> {
    static constexpr bool value = true;
};

// One Stockham pass of radix 2^RLOG after 2^LOGNS points have been combined.
template <int RLOG, int LOGNS, int LOGH, bool INV, class In, class Out>
__device__ __forceinline__ void fft_pass(const In& in, const Out& out, const float2* tw, int tid) {
    constexpr int R = 1 << RLOG;
    constexpr int H = 1 << LOGH;
    constexpr int T = H / 16;
    constexpr int NB = 16 / R;
    constexpr int STR = H / R;
    constexpr int NS = 1 << LOGNS;
    const bool active = tid < T;
    float2 a[16];
    if constexpr (LOGNS == 0 && R == 16 && HasNz<In>::value) {
        // First pass over a zero-padded column: only the points below in.nz() are nonzero, so a
        // warp whose points j + r STR (j >= jw, its first thread) are zero from r = 4 or r = 8
        // on loads and transforms only those (the adjoint sweeps' inputs fill about a fifth of
        // the transform, the forward sweeps' half to three quarters). The choice is uniform
        // over the warp; points beyond a thread's own bound read as zero.
        const int nz = in.nz();
        const int jw = tid & ~31;
        const int rmax = nz <= jw ? 0 : (nz - jw + STR - 1) / STR;
        if (active) {
            if (rmax <= 4) {
#pragma unroll
                for (int r = 0; r < 4; ++r) a[r] = in(tid + r * STR);
                dft16<INV, 4>(a);
            } else if (rmax <= 8) {
#pragma unroll
                for (int r = 0; r < 8; ++r) a[r] = in(tid + r * STR);
                dft16<INV, 8>(a);
            } else {
#pragma unroll
                for (int r = 0; r < 16; ++r) a[r] = in(tid + r * STR);
                dft16<INV>(a);
            }
        }
    } else {
        if (active) {
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const int j = tid + b * T;
#pragma unroll
                for (int r = 0; r < R; ++r) a[b * R + r] = in(j + r * STR);
            }
        }
        if (active) {
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const int j = tid + b * T;
                const int k = j & (NS - 1);
                if constexpr (LOGNS > 0) {
                    // W_{NS R}^{r k} = W_M^{(r k) << (LOGM - LOGNS - RLOG)}, M = 2H
                    constexpr int SH = LOGH + 1 - LOGNS - RLOG;
                    if constexpr (R == 16) {
                        // Two table lookups (w^1, w^4) and at most three complex products for the
                        // other powers: 4 shared loads instead of 30, ~4 ulp per twiddle.
                        float2* x = a + b * R;
                        const float2 w1 = twiddle<LOGH + 1, INV>(tw, k << SH);
                        const float2 w4 = twiddle<LOGH + 1, INV>(tw, (4 * k) << SH);
                        const float2 w2 = cmul(w1, w1);
                        const float2 w3 = cmul(w2, w1);
                        x[1] = cmul(x[1], w1);
                        x[2] = cmul(x[2], w2);
                        x[3] = cmul(x[3], w3);
                        x[4] = cmul(x[4], w4);
                        x[5] = cmul(x[5], cmul(w4, w1));
                        x[6] = cmul(x[6], cmul(w4, w2));
                        x[7] = cmul(x[7], cmul(w4, w3));
                        const float2 w8 = cmul(w4, w4);
                        x[8] = cmul(x[8], w8);
                        x[9] = cmul(x[9], cmul(w8, w1));
                        x[10] = cmul(x[10], cmul(w8, w2));
                        x[11] = cmul(x[11], cmul(w8, w3));
                        const float2 w12 = cmul(w8, w4);
                        x[12] = cmul(x[12], w12);
                        x[13] = cmul(x[13], cmul(w12, w1));
                        x[14] = cmul(x[14], cmul(w12, w2));
                        x[15] = cmul(x[15], cmul(w12, w3));
                    } else {
#pragma unroll
                        for (int r = 1; r < R; ++r)
                            a[b * R + r] = cmul(a[b * R + r], twiddle<LOGH + 1, INV>(tw, (r * k) << SH));
                    }
                }
                dftR<R, INV>(a + b * R);
            }
        }
    }
    // an in-place pass overwrites points other threads read: every load is done before any
    // store (the arithmetic above runs before this barrier, so early warps compute while late
    // ones are still loading)
    if constexpr (In::kSmem && Out::kSmem) __syncthreads();
    if (active) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = tid + b * T;
            const int k = j & (NS - 1);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) out(base + r * NS, a[b * R + r]);
        }
    }
    if constexpr (Out::kSmem) __syncthreads();
}

// W_32^i (forward sign) or its conjugate, i < 8.
template <bool INV, int I>
__device__ __forceinline__ float2 w32c() {
    static_assert(I >= 0 && I < 8, "W_32^i for i < 8");
    // c[i] = cos(2 pi i / 32); sin(2 pi i / 32) = c[8 - i]
    constexpr float c[9] = {1.f, 0.98078528040323044f, 0.92387953251128674f, 0.83146961230254524f,
                            0.70710678118654752f, 0.55557023301960218f, 0.38268343236508978f, 0.19509032201612826f,
                            0.f};
    return make_float2(c[I], INV ? c[8 - I] : -c[8 - I]);
}

// One Stockham pass of radix 32 after NS = 2^LOGNS points have been combined, computed by lane
// pairs: one radix-32 step costs a single shared-memory round trip where a radix-16 and a radix-2
// (or radix-4) pass cost two. The two lanes e = 0, 1 of a pair (group j, twiddle index
// k = j mod NS) hold the even and odd inputs x_{2r+e} (r < 16, input stride H / 32) of the
// group's 32 points. With u = W_{16 NS}^k lane e forms D_e = DFT16(x_{2r+e} u^r), and the 32
// outputs are
//     X[q] = D_0[q] + c_q D_1[q],  X[q + 16] = D_0[q] - c_q D_1[q],  c_q = W_{32 NS}^k W_32^q,  q < 16,
// the odd half's own twiddle W_{32 NS}^k folded into c_q; they go to (j - k) 32 + k + q NS. Lane
// e keeps q in [8e, 8e + 8): it trades the eight D values it does not combine for the partner's
// eight it does (one shuffle each). The partners are lanes l and l ^ 16 (e = bit 4 of the lane,
// j = the other bits), so the sixteen lanes of a half-warp share e and read and write sixteen
// consecutive points of one row: no shared-memory bank conflicts.
template <int LOGNS, int LOGH, bool INV, class In, class Out>
__device__ __forceinline__ void fft_pass32(const In& in, const Out& out, const float2* tw, int tid) {
    constexpr int H = 1 << LOGH;
    constexpr int T = H / 16;
    constexpr int NS = 1 << LOGNS;
    constexpr int STR = H / 32;
    static_assert(LOGNS + 5 <= LOGH, "radix-32 pass within the transform");
    static_assert(T % 32 == 0, "whole warps of lane pairs");
    // u = W_{16 NS}^k = W_M^{k << SU}, W_{32 NS}^k = W_M^{k << (SU - 1)}, M = 2H
    constexpr int SU = LOGH + 1 - LOGNS - 4;
    const bool active = tid < T;
    const int e = (tid >> 4) & 1;
    const int j = (tid & 15) | ((tid >> 5) << 4);
    const int k = j & (NS - 1);
    float2 a[16];
    if (active) {
#pragma unroll
        for (int r = 0; r < 16; ++r) a[r] = in(j + (2 * r + e) * STR);
    }
    if (active) {
        if constexpr (LOGNS > 0) {
            // u^r by the radix-16 pass's scheme: two table values (u, u^4) and products
            const float2 u1 = twiddle<LOGH + 1, INV>(tw, k << SU);
            const float2 u4 = twiddle<LOGH + 1, INV>(tw, (4 * k) << SU);
            const float2 u2 = cmul(u1, u1);
            const float2 u3 = cmul(u2, u1);
            a[1] = cmul(a[1], u1);
            a[2] = cmul(a[2], u2);
            a[3] = cmul(a[3], u3);
            a[4] = cmul(a[4], u4);
            a[5] = cmul(a[5], cmul(u4, u1));
            a[6] = cmul(a[6], cmul(u4, u2));
            a[7] = cmul(a[7], cmul(u4, u3));
            const float2 u8 = cmul(u4, u4);
            a[8] = cmul(a[8], u8);
            a[9] = cmul(a[9], cmul(u8, u1));
            a[10] = cmul(a[10], cmul(u8, u2));
            a[11] = cmul(a[11], cmul(u8, u3));
            const float2 u12 = cmul(u8, u4);
            a[12] = cmul(a[12], u12);
            a[13] = cmul(a[13], cmul(u12, u1));
            a[14] = cmul(a[14], cmul(u12, u2));
            a[15] = cmul(a[15], cmul(u12, u3));
        }
        dft16<INV>(a);
        // lane e = 0 keeps D_0[0..7] and receives D_1[0..7]; lane e = 1 keeps D_1[8..15] and
        // receives D_0[8..15]: afterwards a[i] = D_0[8e + i], a[8 + i] = D_1[8e + i]
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float2 snd = e ? a[i] : a[8 + i];
            float2 rcv;
            rcv.x = __shfl_xor_sync(0xffffffffu, snd.x, 16);
            rcv.y = __shfl_xor_sync(0xffffffffu, snd.y, 16);
            if (e) a[i] = rcv;
            else a[8 + i] = rcv;
        }
        // c_{8e} = W_{32 NS}^k W_32^{8e} = W_M^{(k << (SU - 1)) + e H / 2}; c_{8e + i} = c_{8e} W_32^i.
        // A first pass (k = 0) reads no table: c_{8e} = W_4^e, and a caller may still be filling
        // the table while it runs.
        float2 c0;
        if constexpr (LOGNS == 0) c0 = e ? make_float2(0.f, INV ? 1.f : -1.f) : make_float2(1.f, 0.f);
        else c0 = twiddle<LOGH + 1, INV>(tw, (k << (SU - 1)) + e * (H / 2));
        const float2 cs[8] = {c0,
                              cmul(c0, w32c<INV, 1>()), cmul(c0, w32c<INV, 2>()), cmul(c0, w32c<INV, 3>()),
                              cmul(c0, w32c<INV, 4>()), cmul(c0, w32c<INV, 5>()), cmul(c0, w32c<INV, 6>()),
                              cmul(c0, w32c<INV, 7>())};
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float2 t = cmul(a[8 + i], cs[i]);
            const float2 lo = cadd(a[i], t);
            a[8 + i] = csub(a[i], t);
            a[i] = lo;
        }
    }
    if constexpr (In::kSmem && Out::kSmem) __syncthreads();  // in place: all loads before any store
    if (active) {
        const int base = (j - k) * 32 + k;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int q = 8 * e + i;
            out(base + q * NS, a[i]);
            out(base + (q + 16) * NS, a[8 + i]);
        }
    }
    if constexpr (Out::kSmem) __syncthreads();
}

// Radix (as log2) of the pass after 2^LOGNS of 2^LOGH points have been combined: radix 32 where
// the rest is 5 bits, or 10 bits after a first radix-16 pass (16 + 32 + 32 instead of
// 16 + 16 + 16 + 4 for 2^14 points), else radix 16, else what is left. (2^10 points keep
// 16 + 16 + 4: as 32 + 32 its code is larger, which the persistent multi-length kernel, holding
// every short length at once, pays for in instruction fetch.)
template <int LOGH, int LOGNS>
__host__ __device__ constexpr int fft_rlog() {
    return (LOGH >= 9 && (LOGH - LOGNS == 5 || (LOGNS > 0 && LOGH - LOGNS == 10))) ? 5
           : (LOGNS + 4 <= LOGH)                                                 ? 4
                                                                                 : LOGH - LOGNS;
}

// Passes from LOGNS on; the first one reads through `in`, the last one writes through `out`.
template <int LOGH, bool INV, int LOGNS, class In, class Out>
__device__ __forceinline__ void fft_passes(float2* s, const In& in, const Out& out, const float2* tw, int tid) {
    const SmemPts sp{s};
    constexpr int RLOG = fft_rlog<LOGH, LOGNS>();
    if constexpr (RLOG == 5) {
        if constexpr (LOGNS + 5 == LOGH) {
            fft_pass32<LOGNS, LOGH, INV>(in, out, tw, tid);
        } else {
            fft_pass32<LOGNS, LOGH, INV>(in, sp, tw, tid);
            fft_passes<LOGH, INV, LOGNS + 5>(s, sp, out, tw, tid);
        }
    } else if constexpr (LOGNS + RLOG == LOGH) {
        fft_pass<RLOG, LOGNS, LOGH, INV>(in, out, tw, tid);
    } else {
        fft_pass<RLOG, LOGNS, LOGH, INV>(in, sp, tw, tid);
        fft_passes<LOGH, INV, LOGNS + RLOG>(s, sp, out, tw, tid);
    }
}

// In-place H-point complex FFT (unnormalised) of the padded shared buffer s, with the twiddle
// table of resolution M = 2H in tw (load_twiddles<LOGH + 1>). Must be called by every thread
// of the CTA; the caller syncs before (data and table in shared memory) and may read s after.
template <int LOGH, bool INV>
__device__ __forceinline__ void fft_block(float2* s, const float2* tw) {
    const SmemPts sp{s};
    fft_passes<LOGH, INV, 0>(s, sp, sp, tw, threadIdx.x);
}

// The same transform with the input points read by `in` (z[i], i < H) in the first pass and/or
// the output points handed to `out` (i, Z[i]) by the last pass, so that a global load or store
// is fused into the transform instead of a separate pass over the shared buffer. With a global
// `in` the caller needs no barrier before the call for a twiddle table it filled: the first
// pass uses no twiddles, and its closing barrier publishes the table to the later passes.
template <int LOGH, bool INV, class In, class Out>
__device__ __forceinline__ void fft_block_io(float2* s, const In& in, const Out& out, const float2* tw) {
    fft_passes<LOGH, INV, 0>(s, in, out, tw, threadIdx.x);
}

// Load a real sequence a[0..n) (zero beyond n, up to M = 2H) into s as z[n] = a[2n] + i a[2n+1],
// optionally scaled. The source row must be 8-byte aligned (even element offset).
template <int LOGH>
__device__ __forceinline__ void load_real(float2* s, const float* __restrict__ a, int n, float scale) {
    constexpr int H = 1 << LOGH;
    const float2* a2 = reinterpret_cast<const float2*>(a);
    const int nfull = n >> 1;
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        float2 v;
        if (i < nfull) {
            v = a2[i];
            v.x *= scale;
            v.y *= scale;
        } else if (i == nfull && (n & 1)) {
            v = make_float2(a[n - 1] * scale, 0.f);
        } else {
            v = make_float2(0.f, 0.f);
        }
        s[spad(i)] = v;
    }
}

// Store the first n reals of the unpacked sequence p (p[2i] = Re s[i], p[2i+1] = Im s[i]) times scale.
template <int LOGH>
__device__ __forceinline__ void store_real(const float2* s, float* __restrict__ out, int n, float scale) {
    float2* o2 = reinterpret_cast<float2*>(out);
    const int nfull = n >> 1;
    for (int i = threadIdx.x; i < nfull; i += blockDim.x) {
        float2 v = s[spad(i)];
        o2[i] = make_float2(v.x * scale, v.y * scale);
    }
    if ((n & 1) && threadIdx.x == 0) out[n - 1] = s[spad(nfull)].x * scale;
}

// Real spectrum values A[k] and A[H-k] (k in [1, H/2]) of the packed transform Z held in s:
// A[k] = E + W_M^k O, A[H-k] = conj(E - W_M^k O) with E = (Z_k + conj Z_{H-k})/2,
// O = -i (Z_k - conj Z_{H-k})/2.
template <int LOGH>
__device__ __forceinline__ void unpack_pair(float2 zk, float2 zm, float2 wk, float2& ak, float2& am) {
    float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    // O = -i * (zk - conj zm)/2 ; (zk - conj zm) = (zk.x - zm.x, zk.y + zm.y)
    float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    float2 wo = cmul(wk, o);
    ak = cadd(e, wo);
    am = conjf2(csub(e, wo));
}

// Inverse packing for a Hermitian spectrum P: Z'_k = E' + i O', Z'_{H-k} = conj E' + i conj O'
// with E' = (P_k + conj P_{H-k})/2 and O' = (P_k - conj P_{H-k}) conj(W_M^k)/2.
__device__ __forceinline__ void pack_pair(float2 pk, float2 pm, float2 wk, float2& zk, float2& zm) {
    float2 e = make_float2(0.5f * (pk.x + pm.x), 0.5f * (pk.y - pm.y));
    float2 d = make_float2(0.5f * (pk.x - pm.x), 0.5f * (pk.y + pm.y));
    float2 o = cmulc(d, wk);
    // zk = e + i o ; zm = conj(e) + i conj(o)
    zk = make_float2(e.x - o.y, e.y + o.x);
    zm = make_float2(e.x + o.y, -e.y + o.x);
}

// W_M^k for M = 2^(LOGH+1)
template <int LOGH>
__device__ __forceinline__ float2 wm(const float2* tw, int k) {
    return twiddle<LOGH + 1, false>(tw, k);
}

// Shared-memory floats2 needed for `bufs` transform buffers plus the twiddle table.
template <int LOGH>
__host__ __device__ constexpr int fft_smem_f2(int bufs) {
    return bufs * spad_size(1 << LOGH) + TwSplit<LOGH + 1>::N;
}

}  // namespace ssa
