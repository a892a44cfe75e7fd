"""Pins the NumPy oracle (oracle/ssa_oracle.py) before it is trusted as the checker.

(a) against the reference's own C implementation MKL/ssa_opt_ref.h compiled here
    (oracle/_ref/libssa_ref.so): matvecs, reconstruction, W-correlation, LRF, forecast and
    sequential power iteration on the same inputs / factors;
(b) against the known-answer tests of MKL/test/ssa_opt_test.c;
(c) against the exact dense SVD of the trajectory matrix.
The reference's pure-C randomized SVD (ssa_opt_ref.h:1063-1191) is not used as a pin: on these
inputs it returns non-orthonormal U columns (norms ~1e8), see test_ref_randomized_is_unusable.
"""
import numpy as np
import pytest


def _sig(oracle, N, seed=42):
    return oracle.reference_test_signal(N, seed)


def test_matvec_kat_direct(oracle):
    # MKL/test/ssa_opt_test.c:1464-1508: FFT matvec vs direct sum, N=100, L=25, < 1e-10.
    N, L = 100, 25
    K = N - L + 1
    i = np.arange(N)
    x = np.sin(0.1 * i) + 0.5 * np.cos(0.25 * i)
    v = np.cos(0.05 * np.arange(K))
    assert np.max(np.abs(oracle.hankel_matvec(x, v, L) - oracle.hankel_matvec_direct(x, v, L))) < 1e-10


def test_adjoint_kat_direct(oracle):
    # MKL/test/ssa_opt_test.c:1513-1559.
    N, L = 100, 25
    x = np.sin(0.1 * np.arange(N))
    u = np.cos(0.07 * np.arange(L))
    assert np.max(np.abs(oracle.hankel_matvec_T(x, u, L) - oracle.hankel_matvec_T_direct(x, u, L))) < 1e-10


@pytest.mark.parametrize("N,L", [(100, 25), (500, 125), (1000, 250), (777, 300)])
def test_matvec_short_fft_len(oracle, N, L):
    # The CUDA path uses fft_len = next_pow2(N) instead of next_pow2(N + K - 1): no wrap.
    rng = np.random.default_rng(N)
    x = rng.standard_normal(N)
    K = N - L + 1
    v = rng.standard_normal(K)
    u = rng.standard_normal(L)
    M = oracle.next_pow2(N)
    assert np.allclose(oracle.hankel_matvec(x, v, L, M), oracle.hankel_matvec_direct(x, v, L), atol=1e-10)
    assert np.allclose(oracle.hankel_matvec_T(x, u, L, M), oracle.hankel_matvec_T_direct(x, u, L), atol=1e-10)


def test_matvec_vs_ref(oracle, reflib):
    N, L = 500, 125
    x = _sig(oracle, N)
    K = N - L + 1
    v = np.cos(0.05 * np.arange(K))
    u = np.cos(0.07 * np.arange(L))
    y = np.zeros(L)
    z = np.zeros(K)
    assert reflib.lib.refdrv_matvec(reflib.d(x), N, L, reflib.d(v), reflib.d(y)) == 0
    assert reflib.lib.refdrv_matvec_T(reflib.d(x), N, L, reflib.d(u), reflib.d(z)) == 0
    scale = np.linalg.norm(x) * np.linalg.norm(v)
    assert np.max(np.abs(y - oracle.hankel_matvec(x, v, L))) < 1e-12 * scale
    assert np.max(np.abs(z - oracle.hankel_matvec_T(x, u, L))) < 1e-12 * np.linalg.norm(x) * np.linalg.norm(u)


def _factors(oracle, N, L, k):
    x = _sig(oracle, N)
    d = oracle.dense_svd(x, L, k)
    return x, d, np.ascontiguousarray(d.U.T), np.ascontiguousarray(d.V.T)


@pytest.mark.parametrize("group", [[0], [1, 2], list(range(12)), [0, 99, -1]])
def test_reconstruct_vs_ref(oracle, reflib, group):
    N, L, k = 500, 125, 12
    x, d, Uc, Vc = _factors(oracle, N, L, k)
    g = np.array(group, dtype=np.int32)
    out = np.zeros(N)
    assert reflib.lib.refdrv_reconstruct(reflib.d(x), N, L, k, reflib.d(Uc), reflib.d(Vc), reflib.d(d.sigma),
                                         reflib.i(g), len(g), reflib.d(out)) == 0
    mine = oracle.reconstruct(d, group, N, L)
    assert np.max(np.abs(out - mine)) < 1e-11 * max(1.0, np.max(np.abs(mine)))
    assert np.allclose(mine, oracle.reconstruct_direct(d, group, N, L), atol=1e-9)


def test_wcorr_vs_ref_and_kats(oracle, reflib):
    N, L, k = 500, 125, 12
    x, d, Uc, Vc = _factors(oracle, N, L, k)
    W = np.zeros(k * k)
    assert reflib.lib.refdrv_wcorr(reflib.d(x), N, L, k, reflib.d(Uc), reflib.d(Vc), reflib.d(d.sigma),
                                   reflib.d(W)) == 0
    mine = oracle.wcorr_matrix(d, N, L)
    assert np.max(np.abs(W.reshape(k, k) - mine)) < 1e-12
    # MKL/test/ssa_opt_test.c:411-454: diagonal within 0.01 of 1, symmetric to 1e-10.
    assert np.max(np.abs(np.diag(mine) - 1.0)) < 0.01
    assert np.max(np.abs(mine - mine.T)) < 1e-10
    # wcorr_pair agrees with the matrix (ssa_opt.h:2551-2632).
    assert abs(oracle.wcorr_pair(d, N, L, 1, 2) - mine[1, 2]) < 1e-12


def test_wcorr_elementwise_definition(oracle):
    # W_ij = <x~_i, x~_j>_w / (||x~_i||_w ||x~_j||_w) with w[t] = diagonal counts: the identity
    # the fused CUDA path relies on (elementary reconstructions read by a weighted SYRK).
    N, L, k = 400, 100, 8
    x = _sig(oracle, N, 7)
    d = oracle.dense_svd(x, L, k)
    R = oracle.elementary_reconstructions(d, N, L)
    w = 1.0 / oracle.inv_diag_count(N, L)
    G = R * np.sqrt(w)
    nrm = np.linalg.norm(G, axis=1)
    W = (G @ G.T) / np.outer(nrm, nrm)
    assert np.max(np.abs(W - oracle.wcorr_matrix(d, N, L))) < 1e-10


def test_lrf_forecast_vs_ref(oracle, reflib):
    N, L, k = 500, 125, 12
    x, d, Uc, Vc = _factors(oracle, N, L, k)
    g = np.array([0, 1, 2], dtype=np.int32)
    R = np.zeros(L - 1)
    vert = np.zeros(1)
    assert reflib.lib.refdrv_lrf(reflib.d(x), N, L, k, reflib.d(Uc), reflib.d(Vc), reflib.d(d.sigma),
                                 reflib.i(g), 3, reflib.d(R), reflib.d(vert)) == 0
    R2, nu2 = oracle.compute_lrf(d, [0, 1, 2], L)
    assert np.max(np.abs(R - R2)) < 1e-14
    assert abs(vert[0] - nu2) < 1e-15
    out = np.zeros(N + 30)
    assert reflib.lib.refdrv_forecast(reflib.d(x), N, L, k, reflib.d(Uc), reflib.d(Vc), reflib.d(d.sigma),
                                      reflib.i(g), 3, 30, reflib.d(out)) == 0
    assert np.max(np.abs(out - oracle.forecast_full(d, [0, 1, 2], 30, N, L))) < 1e-9


def test_vforecast_vs_ref_forecast(oracle, reflib):
    """The V-forecast restatement (per-step projections, ssa_opt.h:2906-3084) against the
    reference build's R-forecast on the same factors: the two forms are algebraically equal
    (x_new = sum_g pi_g U_g . z / (1 - nu^2) = R . z), so they agree to FP64 rounding. The
    reference's V-forecast lives in the MKL-only header, so this pins it through that identity."""
    N, L, k = 500, 125, 12
    x, d, Uc, Vc = _factors(oracle, N, L, k)
    g = np.array([0, 1, 2], dtype=np.int32)
    out = np.zeros(N + 30)
    assert reflib.lib.refdrv_forecast(reflib.d(x), N, L, k, reflib.d(Uc), reflib.d(Vc), reflib.d(d.sigma),
                                      reflib.i(g), 3, 30, reflib.d(out)) == 0
    vf = oracle.vforecast_full(d, [0, 1, 2], 30, N, L)
    assert np.max(np.abs(out - vf)) < 1e-9
    # the fast form from the reconstruction is the same forecast
    assert np.max(np.abs(oracle.vforecast_fast(d, [0, 1, 2], vf[:N], 30, L) - vf[N:])) < 1e-9
    with pytest.raises(ValueError):
        oracle.vforecast(d, [0, 99], 5, N, L)


def test_sequential_ref_vs_dense(oracle, reflib):
    N, L, k = 500, 125, 6
    x = _sig(oracle, N)
    K = N - L + 1
    U = np.zeros(L * k)
    V = np.zeros(K * k)
    s = np.zeros(k)
    assert reflib.lib.refdrv_sequential(reflib.d(x), N, L, k, 300, reflib.d(U), reflib.d(V), reflib.d(s)) == k
    d = oracle.dense_svd(x, L, k)
    assert np.max(np.abs(s - d.sigma) / d.sigma) < 2e-3


def test_ref_randomized_is_unusable(oracle, reflib):
    """Documents why ssa_opt_ref.h's randomized SVD is not a pin: its U is not orthonormal."""
    N, L, k, p = 500, 125, 20, 10
    x = _sig(oracle, N)
    K = N - L + 1
    U = np.zeros(L * k)
    V = np.zeros(K * k)
    s = np.zeros(k)
    st = reflib.lib.refdrv_default_state()
    assert reflib.lib.refdrv_randomized(reflib.d(x), N, L, k, p, st, reflib.d(U), reflib.d(V), reflib.d(s)) == k
    norms = np.linalg.norm(U.reshape(k, L), axis=1)
    assert np.max(np.abs(norms - 1.0)) > 1.0


def test_randomized_q0_vs_dense(oracle, reflib):
    # Top components of randomized SVD (q = 0, the reference algorithm) vs the exact SVD.
    N, L, k, p = 1000, 250, 20, 10
    x = _sig(oracle, N)
    K = N - L + 1
    kp = k + p
    Om = np.zeros(K * kp)
    reflib.lib.refdrv_omega(reflib.lib.refdrv_default_state(), K, kp, reflib.d(Om))
    Om = Om.reshape(kp, K).T
    d = oracle.decompose_randomized(x, L, k, p, Om)
    t = oracle.dense_svd(x, L, k)
    assert abs(d.sigma[0] - t.sigma[0]) / t.sigma[0] < 1e-4
    assert np.all(np.diff(d.sigma) <= 0)
    assert np.allclose(d.U.T @ d.U, np.eye(k), atol=1e-12)
    assert np.allclose(d.V.T @ d.V, np.eye(k), atol=1e-12)
    assert np.all(d.U.sum(axis=0) >= 0)


def test_power_iterations_converge(oracle):
    x, clean, Om = oracle.config1(seed=0)
    N, L, k, p = 1000, 250, 50, 10
    t = oracle.dense_svd(x, L, k)
    e0 = np.abs(oracle.decompose_randomized(x, L, k, p, Om, q=0).sigma - t.sigma) / t.sigma
    e2 = np.abs(oracle.decompose_randomized(x, L, k, p, Om, q=2).sigma - t.sigma) / t.sigma
    assert np.max(e2[:3]) < 1e-9
    assert np.mean(e2) < np.mean(e0)


def test_variance_partition(oracle):
    # MKL/test/ssa_opt_test.c:2342-2380: explained variance of all components sums to 1.
    x = _sig(oracle, 500)
    d = oracle.dense_svd(x, 125, 10)
    tot = sum(oracle.variance_explained(d, i, i) for i in range(10))
    assert abs(tot - 1.0) < 1e-3
    assert abs(oracle.variance_explained(d, 0, -1) - 1.0) < 1e-12


def test_block_power_vs_dense(oracle):
    x = _sig(oracle, 500)
    N, L, k = 500, 125, 8
    K = N - L + 1
    rng = np.random.default_rng(5)
    blocks = [rng.uniform(-0.5, 0.5, (K, 4)) for _ in range(2)]
    d = oracle.decompose_block(x, L, k, 4, 100, blocks)
    t = oracle.dense_svd(x, L, k)
    # MKL/test/ssa_opt_test.c:1690-1733: sequential vs block sigma within 1%.
    assert np.max(np.abs(d.sigma - t.sigma) / t.sigma) < 1e-2


def test_mssa_m1_matches_ssa(oracle):
    # MKL/test/ssa_opt_test.c:1857-1892: MSSA with M = 1 equals SSA.
    x = _sig(oracle, 400)
    L, k, p = 100, 6, 8
    K = 400 - L + 1
    Om = np.random.default_rng(1).standard_normal((K, k + p))
    a = oracle.decompose_randomized(x, L, k, p, Om)
    b = oracle.mssa_decompose(x[None, :], L, k, p, Om)
    assert np.allclose(a.sigma, b.sigma, rtol=1e-12)
    assert np.allclose(oracle.reconstruct(a, [0, 1], 400, L), oracle.mssa_reconstruct(b, 0, [0, 1], 1, 400, L))


def _gap_signal(N, two_tones=True):
    """The signals of the reference's gap-filling tests (MKL/test/ssa_opt_test.c:902-1000)."""
    i = np.arange(N, dtype=np.float64)
    s = np.sin(2 * np.pi * i / 50.0) + 0.02 * i
    if two_tones:
        s += 0.5 * np.sin(2 * np.pi * i / 20.0)
    return s


def test_gapfill_reference_bars(oracle):
    """The reference's own acceptance bars: iterative fill of 35 gap values (two runs) leaves no
    NaN and has RMSE < 0.5 at the gaps; the simple form fills a 20-value run."""
    N, L, rank = 500, 100, 6
    true = _gap_signal(N)
    x = true.copy()
    x[50:65] = np.nan
    x[150:170] = np.nan
    om = lambda K, kp: oracle.device_gaussian(oracle.single_series_seed(0), K, kp)  # noqa: E731
    y, it, diff, conv, ng = oracle.gapfill(x, L, rank, 30, 1e-8, om)
    assert ng == 35 and it > 0 and not np.isnan(y).any()
    gaps = np.isnan(x)
    assert np.sqrt(np.mean((y[gaps] - true[gaps]) ** 2)) < 0.5
    assert np.array_equal(y[~gaps], x[~gaps])  # only the gaps change
    t2 = _gap_signal(N, two_tones=False)
    x2 = t2.copy()
    x2[200:220] = np.nan
    y2, ng2 = oracle.gapfill_simple(x2, L, rank, om)
    assert ng2 == 20 and not np.isnan(y2).any()
    assert np.sqrt(np.mean((y2[200:220] - t2[200:220]) ** 2)) < 0.5


def test_gap_linear_start(oracle):
    x = np.array([1.0, np.nan, np.nan, 4.0, np.nan, 6.0, np.nan, np.nan])
    g = np.isnan(x)
    oracle.gap_linear_start(x, g)
    np.testing.assert_allclose(x, [1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 6.0, 6.0])
    y = np.array([np.nan, 2.0])
    oracle.gap_linear_start(y, np.isnan(y))
    assert y[0] == 2.0


def test_parestimate_reference_known_answers(oracle):
    """The oracle's ESPRIT meets the reference's known answers (MKL/test/ssa_opt_test.c:1055-1100,
    2062-2113) on the exact SVD: periods 50 and 20 within 2 samples with moduli > 0.9; periods
    60, 30 and 15 within 5 %."""
    i = np.arange(500, dtype=np.float64)
    x = 3.0 * np.sin(2 * np.pi * i / 50.0) + 2.0 * np.sin(2 * np.pi * i / 20.0)
    r = oracle.parestimate(oracle.dense_svd(x, 125, 6), [0, 1, 2, 3], 125)
    assert any(abs(p - 50.0) < 2.0 for p in r["periods"]) and any(abs(p - 20.0) < 2.0 for p in r["periods"])
    assert all(m > 0.9 for p, m in zip(r["periods"], r["moduli"]) if 5 < p < 100)
    i = np.arange(600, dtype=np.float64)
    x = 4.0 * np.sin(2 * np.pi * i / 60.0) + 2.0 * np.sin(2 * np.pi * i / 30.0) + np.sin(2 * np.pi * i / 15.0)
    r = oracle.parestimate(oracle.dense_svd(x, 150, 8), [0, 1, 2, 3, 4, 5], 150)
    for tp in (60.0, 30.0, 15.0):
        assert min(abs(p - tp) / tp for p, m in zip(r["periods"], r["moduli"]) if m > 0.9) < 0.05
