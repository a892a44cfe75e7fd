"""Parity of the CUDA path (through the C ABI of libssa.so) with the FP64 oracle.

Tolerances (FP32 FFT convolutions and block products, FP64 Gram accumulation / Cholesky /
Rayleigh-Ritz / LRF):
  * matvec: max |y - y_ref| <= 1e-5 * ||x||_2 ||v||_2 (scale-relative; the reference's own KAT
    uses 1e-10 absolute in FP64);
  * singular values: relative error <= SIG_TOL = 1e-5 for every component whose relative gap
    to its neighbours exceeds 1e-3, <= 1e-4 for the rest;
  * reconstructions of groups [0] and [1, 2]: relative L2 <= REC_TOL = 1e-5 when the group's
    singular values are separated from every other computed one by a relative gap > 1e-2;
    otherwise the group is ill-conditioned (its FP32 error is ~ u32 / gap) and the bound is
    max(REC_TOL, 40 * 2^-24 / gap). Signs follow the reference rule sum(U[:, i]) >= 0;
  * W-correlation: max abs <= 1e-4 on the well-separated block, diagonal 1 within 1e-6.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIG_TOL = 1e-5
REC_TOL = 1e-5


@pytest.fixture(scope="module")
def gpu():
    import ssa_gpu

    return ssa_gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def group_gap(sigma, group):
    inside = [i for i in group if 0 <= i < len(sigma)]
    outside = [j for j in range(len(sigma)) if j not in inside]
    if not inside or not outside:
        return np.inf
    return min(abs(sigma[i] - sigma[j]) / sigma[i] for i in inside for j in outside)


def rec_tol(sigma, group):
    g = group_gap(sigma, group)
    return REC_TOL if g > 1e-2 else max(REC_TOL, 40 * 2.0 ** -24 / max(g, 1e-12))


def sigma_errors(s, ref):
    rel = np.abs(s - ref) / ref
    gap = np.full(len(ref), np.inf)
    d = np.abs(np.diff(ref)) / ref[:-1]
    gap[:-1] = np.minimum(gap[:-1], d)
    gap[1:] = np.minimum(gap[1:], d)
    return rel, gap


@pytest.mark.parametrize("N,L", [(100, 25), (4, 2), (5, 3), (31, 10), (33, 32), (777, 300), (1000, 250),
                                 (4096, 1024), (10000, 2500), (20000, 5000), (32768, 8192), (999, 998)])
def test_matvec_vs_direct(gpu, oracle, N, L):
    rng = np.random.default_rng(N + L)
    if N == 100:
        i = np.arange(N)
        x = np.sin(0.1 * i) + 0.5 * np.cos(0.25 * i)  # MKL/test/ssa_opt_test.c:1474-1477
    else:
        x = rng.standard_normal(N) + 0.001 * np.arange(N)
    K = N - L + 1
    v = np.cos(0.05 * np.arange(K)) if N == 100 else rng.standard_normal(K)
    u = rng.standard_normal(L)
    s = gpu.SSA(x, L)
    y = s.hankel_matvec(v)
    z = s.hankel_matvec_T(u)
    yr = oracle.hankel_matvec(x, v, L, oracle.next_pow2(max(N, 32)))
    zr = oracle.hankel_matvec_T(x, u, L, oracle.next_pow2(max(N, 32)))
    assert np.max(np.abs(y - yr)) <= 1e-5 * np.linalg.norm(x) * np.linalg.norm(v)
    assert np.max(np.abs(z - zr)) <= 1e-5 * np.linalg.norm(x) * np.linalg.norm(u)


@pytest.mark.parametrize("q", [0, 2])
def test_config1_parity_host_omega(gpu, oracle, q):
    x, clean, Om = oracle.config1(seed=0)
    N, L, k, p = 1000, 250, 50, 10
    d = oracle.decompose_randomized(x, L, k, p, Om, q=q)
    gs = gpu.SSA(x, L)
    gs.decompose(k, oversampling=p, power_iters=q, omega=Om)
    U, V, s = gs.factors()
    rel, gap = sigma_errors(s, d.sigma)
    sep = gap > 1e-3
    print(f"\nq={q}: max sigma rel err {rel.max():.2e} (separated {rel[sep].max():.2e})")
    assert np.all(rel[sep] <= SIG_TOL)
    assert np.all(rel <= 1e-4)
    assert np.max(np.abs(U.T @ U - np.eye(k))) < 1e-4
    for g in ([0], [1, 2]):
        e = rel_l2(gs.reconstruct(g), oracle.reconstruct(d, g, N, L))
        print(f"  group {g}: rel L2 {e:.2e}")
        assert e <= REC_TOL
    W = gs.wcorr_matrix()
    Wr = oracle.wcorr_matrix(d, N, L)
    print(f"  W max abs err {np.max(np.abs(W - Wr)):.2e}")
    assert np.max(np.abs(np.diag(W) - 1.0)) < 1e-6
    assert np.max(np.abs(W[:5, :5] - Wr[:5, :5])) < 1e-4


def test_device_generator_matches_replica(gpu, oracle):
    x, clean, _ = oracle.config1(seed=0)
    N, L, k, p = 1000, 250, 20, 10
    K = N - L + 1
    gs = gpu.SSA(x, L)
    gs.decompose(k, oversampling=p)  # q = 0, generated Omega, first draw of this context
    Om = oracle.device_gaussian(oracle.single_series_seed(0), K, k + p)
    d = oracle.decompose_randomized(x, L, k, p, Om, q=0)
    rel, gap = sigma_errors(gs.singular_values, d.sigma)
    assert np.all(rel[gap > 1e-3] <= SIG_TOL)
    assert rel_l2(gs.reconstruct([0]), oracle.reconstruct(d, [0], N, L)) <= REC_TOL


def test_q2_vs_dense_truth(gpu, oracle):
    x, clean, Om = oracle.config1(seed=0)
    N, L, k, p = 1000, 250, 50, 10
    t = oracle.dense_svd(x, L, k)
    gs = gpu.SSA(x, L)
    gs.decompose(k, oversampling=p, power_iters=2, omega=Om)
    s = gs.singular_values
    # leading components converge to the exact SVD with q = 2 (oracle: <= 1e-9 for 3 components)
    assert np.max(np.abs(s[:3] - t.sigma[:3]) / t.sigma[:3]) <= SIG_TOL
    assert rel_l2(gs.reconstruct([0]), oracle.reconstruct(t, [0], N, L)) <= REC_TOL


def test_forecast_parity(gpu, oracle):
    x, clean, Om = oracle.config1(seed=0)
    N, L, k, p = 1000, 250, 10, 10
    d = oracle.decompose_randomized(x, L, k, p, Om[:, :k + p], q=2)
    gs = gpu.SSA(x, L)
    gs.decompose(k, oversampling=p, power_iters=2, omega=Om[:, :k + p])
    g = [0, 1, 2]
    R, nu2 = gs.lrf(g)
    Rr, nu2r = oracle.compute_lrf(d, g, L)
    assert abs(nu2 - nu2r) < 1e-5
    assert rel_l2(R, Rr) < 1e-4
    f = gs.forecast(g, 50)
    fr = oracle.forecast(d, g, 50, N, L)
    assert rel_l2(f, fr) < 1e-4
    full = gs.forecast_full(g, 20)
    assert rel_l2(full[:N], oracle.reconstruct(d, g, N, L)) <= REC_TOL
    assert rel_l2(full[N:], fr[:20]) < 1e-4


def test_vforecast_parity(gpu, oracle):
    """V-forecast (ssa_opt_vforecast*, MKL/ssa_opt.h:2906-3084) against the oracle's per-step
    projection form, same tolerances as the R-forecast; the V and R forms agree to FP64 rounding."""
    x, clean, Om = oracle.config1(seed=0)
    N, L, k, p = 1000, 250, 10, 10
    d = oracle.decompose_randomized(x, L, k, p, Om[:, :k + p], q=2)
    gs = gpu.SSA(x, L)
    gs.decompose(k, oversampling=p, power_iters=2, omega=Om[:, :k + p])
    g = [0, 1, 2]
    fr = oracle.vforecast(d, g, 50, N, L)
    np.testing.assert_allclose(fr, oracle.forecast(d, g, 50, N, L), rtol=1e-10, atol=1e-10 * np.abs(fr).max())
    f = gs.vforecast(g, 50)
    assert rel_l2(f, fr) < 1e-4
    np.testing.assert_allclose(f, gs.forecast(g, 50), rtol=1e-12, atol=0)
    full = gs.vforecast_full(g, 20)
    assert rel_l2(full[:N], oracle.reconstruct(d, g, N, L)) <= REC_TOL
    assert rel_l2(full[N:], fr[:20]) < 1e-4
    # from a caller's base signal: the clean signal (any length >= L - 1), and the raw series
    for base in (clean, x[:600]):
        fb = gs.vforecast_fast(g, base, 30)
        fbr = oracle.vforecast_fast(d, g, base, 30, L)
        assert rel_l2(fb, fbr) < 1e-4
    # from the group's own reconstruction it is the V-forecast itself
    np.testing.assert_allclose(gs.vforecast_fast(g, full[:N], 20), f[:20], rtol=1e-9,
                               atol=1e-9 * np.abs(f).max())
    with pytest.raises(RuntimeError):
        gs.vforecast_fast(g, x[:L - 2], 5)  # base shorter than L - 1
    with pytest.raises(RuntimeError):
        gs.vforecast([0, 99], 5)  # index outside the decomposition


def test_extend_matches_exact_svd(gpu, oracle):
    """ssa_opt_extend (MKL/ssa_opt.h:1935-2056): components added to a randomized decomposition by
    deflated one-column power iterations reach the exact SVD's (sigma within 1e-5 relative for
    well-separated values; U columns within 5e-4 up to sign: FP32 iterates, and a singular
    vector's error grows as 1/gap, 1e-4 measured at gaps of a few percent), all re-sorted by
    sigma; the new
    components follow the sign rule, the old ones keep theirs."""
    x, _, Om = oracle.config1(seed=0)
    N, L = 1000, 250
    t = oracle.dense_svd(x, L, 12)
    gs = gpu.SSA(x, L)
    gs.decompose(4, oversampling=10, power_iters=2, omega=Om[:, :14])
    U0, _, _ = gs.factors()
    gs.extend(3, max_iter=200)
    assert gs.n_components == 7
    s = gs.singular_values
    assert np.all(np.diff(s) <= 0)
    U, V, _ = gs.factors()
    for i in range(7):
        gap = min(abs(t.sigma[i] - t.sigma[j]) / t.sigma[i] for j in range(12) if j != i)
        if gap > 1e-2:
            assert abs(s[i] - t.sigma[i]) / t.sigma[i] <= 1e-5, i
            d = min(np.linalg.norm(U[:, i] - t.U[:, i]), np.linalg.norm(U[:, i] + t.U[:, i]))
            assert d <= 5e-4, (i, d)
    assert np.all(U[:, 4:].sum(axis=0) >= 0)
    np.testing.assert_array_equal(U[:, :4], U0)  # the old factors are kept as they were
    # the largest leading group that does not split a near-degenerate pair (boundary gap > 1e-2)
    m = max(j for j in range(1, 8) if abs(t.sigma[j - 1] - t.sigma[j]) / t.sigma[j - 1] > 1e-2)
    assert m >= 4
    assert rel_l2(gs.reconstruct(list(range(m))), oracle.reconstruct(t, list(range(m)), N, L)) <= 1e-4
    with pytest.raises(RuntimeError):
        gs.extend(100, max_iter=5)  # beyond the 64-column capacity of the context
    with pytest.raises(RuntimeError):
        gpu.SSA(x, L).extend(2)  # nothing decomposed yet


def test_reconstruct_edge_groups(gpu, oracle):
    x, _, Om = oracle.config1(seed=0)
    N, L, k, p = 1000, 250, 8, 4
    d = oracle.decompose_randomized(x, L, k, p, Om[:, :k + p], q=1)
    gs = gpu.SSA(x, L)
    gs.decompose(k, oversampling=p, power_iters=1, omega=Om[:, :k + p])
    # out-of-range indices are skipped (MKL/ssa_opt.h:2347-2348)
    assert rel_l2(gs.reconstruct([0, 99, -3]), oracle.reconstruct(d, [0], N, L)) <= REC_TOL
    assert np.all(gs.reconstruct([50]) == 0.0)
    # full group = sum of all components
    assert rel_l2(gs.reconstruct(list(range(k))), oracle.reconstruct(d, list(range(k)), N, L)) <= REC_TOL
    # get_trend / get_noise
    assert rel_l2(gs.get_trend(), oracle.reconstruct(d, [0], N, L)) <= REC_TOL
    assert rel_l2(gs.get_noise(3), oracle.reconstruct(d, list(range(3, k)), N, L)) <= 1e-4
    assert np.all(gs.get_noise(k) == 0.0)
    with pytest.raises(RuntimeError):
        gs.reconstruct([])
    # cached spectra give the same values
    a = gs.reconstruct([1, 2])
    gs.cache_ffts()
    assert np.array_equal(a, gs.reconstruct([1, 2]))


def test_api_errors(gpu, oracle):
    x = oracle.reference_test_signal(1000)
    with pytest.raises(ValueError):
        gpu.SSA(x[:3], 2)
    with pytest.raises(ValueError):
        gpu.SSA(x, 1)
    with pytest.raises(ValueError):
        gpu.SSA(x, 1000)
    with pytest.raises(ValueError):
        gpu.SSA(np.zeros(140000), 100)  # beyond the largest FFT length (N <= 131072)
    s = gpu.SSA(x, 250)
    with pytest.raises(RuntimeError):
        s.reconstruct([0])
    with pytest.raises(RuntimeError):
        s.decompose(60, oversampling=10)  # k + p > SSA_MAX_KP
    s.decompose(5, oversampling=5)
    with pytest.raises(RuntimeError):
        s.forecast([0, 7], 5)  # out-of-range index in the LRF group (MKL/ssa_opt.h:2781-2785)
    assert s.wcorr(0, 99) == 0.0
    assert s.variance_explained(0, -1) == pytest.approx(1.0)


def test_update_signal_and_repeat(gpu, oracle):
    x, _, Om = oracle.config1(seed=0)
    y, _, _ = oracle.config1(seed=5)
    N, L, k, p = 1000, 250, 10, 6
    s = gpu.SSA(x, L)
    s.decompose(k, oversampling=p, power_iters=2, omega=Om[:, :k + p])
    s.update_signal(y)
    with pytest.raises(RuntimeError):
        s.reconstruct([0])
    s.decompose(k, oversampling=p, power_iters=2, omega=Om[:, :k + p])
    d = oracle.decompose_randomized(y, L, k, p, Om[:, :k + p], q=2)
    rel, gap = sigma_errors(s.singular_values, d.sigma)
    assert np.all(rel[gap > 1e-3] <= SIG_TOL)


def test_constant_signal(gpu):
    # MKL/test/ssa_opt_test.c:1289-1322: rank-1 trajectory matrix.
    x = np.full(300, 5.0)
    s = gpu.SSA(x, 75)
    s.decompose(5, oversampling=5)
    sv = s.singular_values
    assert sv[0] == pytest.approx(5.0 * np.sqrt(75 * 226), rel=1e-5)
    assert np.all(sv[1:] < 1e-4 * sv[0])
    assert np.max(np.abs(s.reconstruct([0]) - 5.0)) < 1e-4


def test_batch_matches_single_and_oracle(gpu, oracle):
    B, N, L, k, p, q = 6, 2000, 500, 20, 10, 2
    X = oracle.config2_batch(B, seed=11, N=N)
    b = gpu.SSABatch(B, N, L, k, oversampling=p, power_iters=q, groups=[[0], [1, 2]])
    sig, W, G = b.run(X, seed=123)
    # batch invariance: series 0 alone in the same engine gives the same bits as in the mix
    sig0, W0, G0 = b.run(X[0:1], seed=123)
    assert np.array_equal(sig0[0], sig[0])
    assert np.array_equal(G0[0], G[0])
    assert np.array_equal(W0[0], W[0])
    for s_ in range(B):
        Om = oracle.device_gaussian(oracle.series_seed(123, s_), N - L + 1, k + p)
        d = oracle.decompose_randomized(X[s_], L, k, p, Om, q=q)
        rel, gap = sigma_errors(sig[s_], d.sigma)
        assert np.all(rel[gap > 1e-3] <= SIG_TOL), (s_, rel.max())
        assert rel_l2(G[s_, 0], oracle.reconstruct(d, [0], N, L)) <= rec_tol(d.sigma, [0])
        assert rel_l2(G[s_, 1], oracle.reconstruct(d, [1, 2], N, L)) <= rec_tol(d.sigma, [1, 2])
        assert np.max(np.abs(np.diag(W[s_]) - 1.0)) < 1e-6


def test_kernel_launch_counter(gpu, oracle):
    before = gpu.kernel_launches()
    s = gpu.SSA(oracle.reference_test_signal(500), 125)
    s.decompose(10)
    s.reconstruct([0])
    assert gpu.kernel_launches() > before


def _device_checks(gpu):
    import ctypes
    chk = (ctypes.c_uint * 5)()
    assert gpu._lib.ssa_b200_device_checks(chk, 1) == 0
    return list(chk)


def test_full_size_batch_clean(gpu, oracle):
    """Uniform-batch sizes (N = 10000, L = 2500, k = 50, p = 10, q = 2) over 256 series: every
    series succeeds, the kernels' self-checks record nothing, and two series match the oracle."""
    import torch

    B, N, L, k, p, q = 256, 10000, 2500, 50, 10, 2
    _device_checks(gpu)
    X = oracle.config2_batch(B, seed=3, N=N)
    d_x = torch.from_numpy(X).cuda()
    b = gpu.SSABatch(B, N, L, k, oversampling=p, power_iters=q, groups=[[0], [1, 2]])
    for seed in (5, 6):
        b.run_device(d_x.data_ptr(), B, seed=seed)
        b.sync()
    assert np.count_nonzero(b.status(B)) == 0
    assert _device_checks(gpu)[0] == 0
    sig, W, G = b.run(X, seed=6)
    for s_ in (0, B - 1):
        Om = oracle.device_gaussian(oracle.series_seed(6, s_), N - L + 1, k + p)
        d = oracle.decompose_randomized(X[s_], L, k, p, Om, q=q)
        rel, gap = sigma_errors(sig[s_], d.sigma)
        assert np.all(rel[gap > 1e-3] <= SIG_TOL), (s_, rel.max())
        assert rel_l2(G[s_, 1], oracle.reconstruct(d, [1, 2], N, L)) <= rec_tol(d.sigma, [1, 2])


@pytest.mark.parametrize("k,bsize,max_iter", [(10, 4, 20), (6, 6, 30), (8, 3, 7)])
def test_block_power_parity(gpu, oracle, k, bsize, max_iter):
    """Block power iteration (MKL/ssa_opt.h:1765-1933) with the same start blocks as the oracle.
    The device re-orthonormalises every half-step (the reference every fifth); the subspaces,
    hence the Rayleigh-Ritz results, are the same."""
    x, _, _ = oracle.config1(seed=0)
    N, L = 1000, 250
    K = N - L + 1
    rng = np.random.default_rng(k * 100 + bsize)
    V0 = rng.uniform(-0.5, 0.5, (K, k))
    blocks, c = [], 0
    while c < k:
        cb = min(bsize, k - c)
        blocks.append(V0[:, c:c + cb])
        c += cb
    d = oracle.decompose_block(x, L, k, bsize, max_iter, blocks)
    gs = gpu.SSA(x, L)
    gs.decompose(k, method="block", block_size=bsize, max_iter=max_iter, v0=V0)
    U, V, s = gs.factors()
    rel, gap = sigma_errors(s, d.sigma)
    assert np.all(rel[gap > 1e-3] <= SIG_TOL), rel.max()
    assert np.all(rel <= 1e-4)
    for g in ([0], [1, 2]):
        assert rel_l2(gs.reconstruct(g), oracle.reconstruct(d, g, N, L)) <= rec_tol(d.sigma, g)


def test_sequential_and_block_agree_with_exact(gpu, oracle):
    # MKL/test/ssa_opt_test.c:1690-1733: methods agree within 1%; here also vs the exact SVD.
    x = oracle.reference_test_signal(500)
    N, L, k = 500, 125, 6
    t = oracle.dense_svd(x, L, k)
    a = gpu.SSA(x, L)
    a.decompose(k, method="sequential", max_iter=100)
    b = gpu.SSA(x, L)
    b.decompose(k, method="block", block_size=3, max_iter=100)
    sa, sb = a.singular_values, b.singular_values
    assert np.max(np.abs(sa - sb) / sb) < 1e-2
    assert np.max(np.abs(sb - t.sigma) / t.sigma) < 1e-2
    assert np.abs(sb[0] - t.sigma[0]) / t.sigma[0] < 1e-5
    assert np.all(np.diff(sb) <= 0)
    U, V, _ = b.factors()
    assert np.all(U.sum(axis=0) >= 0)


def test_context_recycling_same_results_and_bounded_memory(gpu, oracle):
    """Contexts created with recycling (streams, pooled device buffers and page-locked staging of
    freed contexts) give bit-identical results to freshly allocated ones, and creating and freeing
    contexts per series keeps device memory bounded (the pool reuses its cached blocks)."""
    import torch

    x, _, Om = oracle.config1(seed=2)
    d = oracle.decompose_randomized(x, 250, 20, 10, Om, q=2)
    got = []
    try:
        for on in (False, True, True, False):
            gpu.set_context_recycling(on)
            s = gpu.SSA(x, 250)
            s.decompose(20, oversampling=10, power_iters=2, omega=Om)
            got.append((s.singular_values.copy(), s.reconstruct([0, 1]), s.wcorr_matrix()))
            del s
        for sg, rec, W in got[1:]:
            assert np.array_equal(sg, got[0][0]) and np.array_equal(rec, got[0][1]) and np.array_equal(W, got[0][2])
        assert np.max(np.abs(got[0][0][:3] - d.sigma[:3]) / d.sigma[:3]) < 1e-5
        gpu.set_context_recycling(True)
        rng = np.random.default_rng(5)
        shapes = [(1000, 250, 20), (7000, 1750, 40), (30000, 7500, 30)]
        series = [(rng.standard_normal(N).cumsum(), L, k) for N, L, k in shapes]

        def cycle(n):
            for i in range(n):
                xs, L, k = series[i % 3]
                s = gpu.SSA(xs, L)
                s.decompose(k, oversampling=10, power_iters=1)
                s.reconstruct([0])
                del s

        cycle(6)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        cycle(60)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert free0 - free1 < 64 << 20, (free0, free1)
    finally:
        gpu.set_context_recycling(True)
