/* Known-answer acceptance program for the drop-in C API, built against include/ssa_opt.h and
 * linked with libssa.so exactly as a C caller of the reference library would be.
 *
 * It runs the checks the reference's own C tests make on this path, in this program's own code:
 *   - FFT matvec / adjoint against direct sums (MKL/test/ssa_opt_test.c:1464-1559), through the
 *     reference-named ssa_opt_hankel_matvec / _T; bar 1e-5 * |x| |v| (the device runs FP32; the
 *     reference's FP64 bar is 1e-10 absolute);
 *   - singular values positive and descending after a randomized decomposition (:188-280),
 *     read directly from the host-visible struct fields (sigma, n_components, U, V);
 *   - W-correlation symmetric, unit diagonal, a sine/cosine pair correlated above 0.5
 *     (:411-454), and the same matrix after ssa_opt_cache_ffts (fast vs slow, :1192-1232);
 *   - variance partition: the per-component shares sum to the whole (:2342-2380);
 *   - block and randomized decompositions agree on the leading singular values within 1%
 *     (:1690-1733);
 *   - forecast of a trend+cycles signal follows the continuation (correlation > 0.8, :493-532).
 * Exit status 0 when every check passes; one line per check on stdout.
 * Build: gcc -O2 -I include tests/c/kat_drop_in.c -L<dir of libssa.so> -lssa -lm */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ssa_opt.h"

static int g_fail = 0;

static void check(int ok, const char *what, double value)
{
    printf("%s %-58s %.3e\n", ok ? "PASS" : "FAIL", what, value);
    if (!ok)
        g_fail = 1;
}

/* deterministic test signal: trend + two cycles (periods 100 and 25) + uniform-sum noise */
static void test_signal(double *x, int n, unsigned long long seed)
{
    unsigned long long s = seed * 0x9E3779B97F4A7C15ull + 1;
    for (int i = 0; i < n; i++) {
        double noise = 0.0;
        for (int r = 0; r < 4; r++) {
            s ^= s << 13;
            s ^= s >> 7;
            s ^= s << 17;
            noise += (double)(s >> 11) / 9007199254740992.0 - 0.5;
        }
        const double t = (double)i / n;
        x[i] = 100.0 + 50.0 * t + 20.0 * sin(2.0 * M_PI * i / 100.0) + 10.0 * sin(2.0 * M_PI * i / 25.0) +
               3.0 * noise;
    }
}

static void kat_matvec(void)
{
    const int N = 100, L = 25, K = N - L + 1;
    double x[100], v[76], u[25], y[25], z[76];
    for (int i = 0; i < N; i++)
        x[i] = sin(0.1 * i) + 0.5 * cos(0.25 * i);
    for (int j = 0; j < K; j++)
        v[j] = cos(0.05 * j);
    for (int i = 0; i < L; i++)
        u[i] = cos(0.07 * i);
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0) {
        check(0, "init N=100 L=25", 0);
        return;
    }
    ssa_opt_hankel_matvec(&s, v, y);
    ssa_opt_hankel_matvec_T(&s, u, z);
    double ex = 0, ez = 0, nx = 0, nv = 0, nu = 0;
    for (int i = 0; i < N; i++)
        nx += x[i] * x[i];
    for (int j = 0; j < K; j++)
        nv += v[j] * v[j];
    for (int i = 0; i < L; i++)
        nu += u[i] * u[i];
    for (int i = 0; i < L; i++) {
        double d = 0;
        for (int j = 0; j < K; j++)
            d += x[i + j] * v[j];
        ex = fmax(ex, fabs(d - y[i]));
    }
    for (int j = 0; j < K; j++) {
        double d = 0;
        for (int i = 0; i < L; i++)
            d += x[i + j] * u[i];
        ez = fmax(ez, fabs(d - z[j]));
    }
    check(ex <= 1e-5 * sqrt(nx * nv), "matvec vs direct sum (N=100, L=25)", ex);
    check(ez <= 1e-5 * sqrt(nx * nu), "adjoint matvec vs direct sum (N=100, L=25)", ez);
    ssa_opt_free(&s);
}

static void kat_decomposition(void)
{
    const int N = 1000, L = 250, k = 12;
    double *x = malloc(sizeof(double) * N);
    test_signal(x, N, 7);
    SSA_Opt s;
    if (ssa_opt_init(&s, x, N, L) != 0 || ssa_opt_prepare(&s, k, 8) != 0 ||
        ssa_opt_decompose_randomized(&s, k, 8) != 0) {
        check(0, "randomized decomposition", 0);
        free(x);
        return;
    }
    int sorted = s.n_components == k && s.sigma[k - 1] > 0;
    for (int i = 1; i < s.n_components; i++)
        sorted &= s.sigma[i] <= s.sigma[i - 1];
    check(sorted, "sigma > 0 and descending (host struct fields)", s.sigma[0]);
    double orth = 0;
    for (int a = 0; a < k; a++)
        for (int b = 0; b < k; b++) {
            double d = 0;
            for (int t = 0; t < L; t++)
                d += s.U[a * L + t] * s.U[b * L + t];
            orth = fmax(orth, fabs(d - (a == b)));
        }
    check(orth < 1e-4, "U columns orthonormal (host struct field U)", orth);

    double *W = malloc(sizeof(double) * k * k), *W2 = malloc(sizeof(double) * k * k);
    int ok = ssa_opt_wcorr_matrix(&s, W) == 0;
    double diag = 0, sym = 0;
    for (int i = 0; i < k; i++) {
        diag = fmax(diag, fabs(W[i * k + i] - 1.0));
        for (int j = 0; j < k; j++)
            sym = fmax(sym, fabs(W[i * k + j] - W[j * k + i]));
    }
    check(ok && diag < 0.01, "W diagonal within 0.01 of 1", diag);
    check(ok && sym < 1e-10, "W symmetric", sym);
    check(ok && fabs(W[1 * k + 2]) > 0.5, "W(1,2) of the period-100 pair > 0.5", fabs(W[1 * k + 2]));
    ok = ssa_opt_cache_ffts(&s) == 0 && ssa_opt_wcorr_matrix_fast(&s, W2) == 0;
    double fs = 0;
    for (int i = 0; i < k * k; i++)
        fs = fmax(fs, fabs(W[i] - W2[i]));
    check(ok && fs < 1e-6, "W with cached spectra equals W without (fast vs slow)", fs);

    double parts = 0;
    for (int i = 0; i < k; i++)
        parts += ssa_opt_variance_explained(&s, i, i);
    const double whole = ssa_opt_variance_explained(&s, 0, -1);
    check(fabs(parts - whole) < 1e-3 && fabs(whole - 1.0) < 1e-9, "variance partition", fabs(parts - whole));

    double sig_r[3];
    memcpy(sig_r, s.sigma, sizeof(sig_r));
    if (ssa_opt_decompose_block(&s, 6, 6, 100) != 0) {
        check(0, "block decomposition", 0);
    } else {
        double rel = 0;
        for (int i = 0; i < 3; i++)
            rel = fmax(rel, fabs(s.sigma[i] - sig_r[i]) / sig_r[i]);
        check(rel < 0.01, "block vs randomized leading sigma within 1%", rel);
    }
    free(W);
    free(W2);
    ssa_opt_free(&s);
    free(x);
}

static void kat_forecast(void)
{
    const int N = 1200, L = 200, h = 100;
    double *full = malloc(sizeof(double) * (N + h)), *fc = malloc(sizeof(double) * h);
    for (int i = 0; i < N + h; i++)
        full[i] = 10.0 + 0.01 * i + 5.0 * sin(2.0 * M_PI * i / 40.0) + 2.0 * sin(2.0 * M_PI * i / 15.0);
    SSA_Opt s;
    const int g[5] = {0, 1, 2, 3, 4};
    if (ssa_opt_init(&s, full, N, L) != 0 || ssa_opt_prepare(&s, 8, 8) != 0 ||
        ssa_opt_decompose_randomized(&s, 8, 8) != 0 || ssa_opt_forecast(&s, g, 5, h, fc) != 0) {
        check(0, "forecast", 0);
    } else {
        double ma = 0, mb = 0, sab = 0, saa = 0, sbb = 0;
        for (int i = 0; i < h; i++) {
            ma += fc[i] / h;
            mb += full[N + i] / h;
        }
        for (int i = 0; i < h; i++) {
            sab += (fc[i] - ma) * (full[N + i] - mb);
            saa += (fc[i] - ma) * (fc[i] - ma);
            sbb += (full[N + i] - mb) * (full[N + i] - mb);
        }
        const double corr = sab / sqrt(saa * sbb + 1e-300);
        check(corr > 0.8, "forecast correlates with the continuation", corr);
    }
    ssa_opt_free(&s);
    free(full);
    free(fc);
}

int main(void)
{
    printf("sizeof(SSA_Opt) = %zu bytes\n", sizeof(SSA_Opt));
    kat_matvec();
    kat_decomposition();
    kat_forecast();
    printf("%s\n", g_fail ? "FAILED" : "ALL PASSED");
    return g_fail;
}
