"""Series longer than 32768 (FFT lengths 65536 and 131072, run on thread-block clusters) against
the FP64 oracle: matvecs, decomposition, grouped and elementary reconstructions, W-correlation,
and an uneven batch across single-CTA and cluster FFT lengths.

Tolerances as in the single-series parity tests: matvec max |y - y_ref| <= 1e-5 ||x|| ||v||;
singular values relative <= 1e-5 where the relative gap exceeds 1e-3 (1e-4 otherwise);
reconstructions relative L2 <= 1e-5 for groups separated by a relative gap > 1e-2, else
max(1e-5, 40 * 2^-24 / gap); W-correlation diagonal within 1e-6, leading separated block 1e-4.
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


def check_sigma(s, ref):
    rel = np.abs(s - ref) / ref
    gap = np.full(len(ref), np.inf)
    d = np.abs(np.diff(ref)) / ref[:-1]
    gap[:-1] = np.minimum(gap[:-1], d)
    gap[1:] = np.minimum(gap[1:], d)
    assert np.all(rel[gap > 1e-3] <= SIG_TOL), rel.max()
    assert np.all(rel <= 1e-4), rel.max()


@pytest.mark.parametrize("N,L", [(40000, 10000), (65536, 16384), (100000, 25000), (131072, 100), (131072, 131000)])
def test_large_matvec_vs_direct(gpu, oracle, N, L):
    rng = np.random.default_rng(N + L)
    x = rng.standard_normal(N) + 0.001 * np.arange(N)
    K = N - L + 1
    v = rng.standard_normal(K)
    u = rng.standard_normal(L)
    s = gpu.SSA(x, L)
    y = s.hankel_matvec(v)
    z = s.hankel_matvec_T(u)
    M = oracle.next_pow2(N)
    yr = oracle.hankel_matvec(x, v, L, M)
    zr = oracle.hankel_matvec_T(x, u, L, M)
    assert np.max(np.abs(y - yr)) <= 1e-5 * np.linalg.norm(x) * np.linalg.norm(v)
    assert np.max(np.abs(z - zr)) <= 1e-5 * np.linalg.norm(x) * np.linalg.norm(u)


@pytest.mark.parametrize("N", [50000, 100000])
def test_large_decompose_reconstruct_wcorr(gpu, oracle, N):
    rng = np.random.default_rng(N)
    x = oracle.walk_sines(rng, N)
    L, k, p = N // 4, 12, 10
    K = N - L + 1
    Om = rng.standard_normal((K, k + p))
    d = oracle.decompose_randomized(x, L, k, p, Om, q=2)
    s = gpu.SSA(x, L)
    s.decompose(k, oversampling=p, power_iters=2, omega=Om)
    check_sigma(s.singular_values, d.sigma)
    for g in ([0], [1, 2], [0, 1, 2, 3]):
        e = rel_l2(s.reconstruct(g), oracle.reconstruct(d, g, N, L))
        assert e <= rec_tol(d.sigma, g), (g, e)
    W = s.wcorr_matrix()
    Wr = oracle.wcorr_matrix(d, N, L)
    assert np.max(np.abs(np.diag(W) - 1.0)) < 1e-6
    blk = [i for i in range(min(6, k)) if group_gap(d.sigma, [i]) > 1e-2]
    assert blk and np.max(np.abs(W[np.ix_(blk, blk)] - Wr[np.ix_(blk, blk)])) < 1e-4
    fc = s.forecast([0, 1, 2], 30)
    fr = oracle.forecast(d, [0, 1, 2], 30, N, L)
    assert rel_l2(fc, fr) <= 1e-4


def test_uneven_batch_across_cluster_lengths(gpu, oracle):
    rng = np.random.default_rng(3)
    mix = [(oracle.walk_sines(rng, N), N // 4, k) for N, k in
           ((900, 20), (40000, 15), (20000, 30), (100000, 12), (70000, 25), (5000, 40))]
    p, q, seed = 10, 2, 17
    rb = gpu.SSARaggedBatch(oversampling=p, power_iters=q, groups=[[0], [1, 2]])
    sig, W, G = rb.run([m[0] for m in mix], [m[1] for m in mix], [m[2] for m in mix], seed=seed)
    for s, (x, L, k) in enumerate(mix):
        N = len(x)
        K = N - L + 1
        Om = oracle.device_gaussian(oracle.series_seed(seed, s), K, min(k + p, L, K))
        d = oracle.decompose_randomized(x, L, k, p, Om, q=q)
        check_sigma(sig[s], d.sigma)
        for gi, g in enumerate(([0], [1, 2])):
            assert rel_l2(G[s][gi], oracle.reconstruct(d, g, N, L)) <= rec_tol(d.sigma, g), (s, N, g)
        assert np.max(np.abs(np.diag(W[s]) - 1.0)) < 1e-6


def test_uneven_batch_mixed_radix_boundaries(gpu, oracle):
    """Both sides of the mixed-radix FFT lengths (real lengths 49152, 81920 and 98304, clusters of
    3, 5 and 6 CTAs) against the oracle: 32769 and 49152 run at 49152, 49153 at 65536, 65537 and
    81920 at 81920, 81921 and 98304 at 98304, 98305 at 131072."""
    rng = np.random.default_rng(11)
    mix = [(oracle.walk_sines(rng, N), N // 4, k) for N, k in
           ((32769, 14), (49152, 22), (49153, 10), (65537, 12), (81920, 16), (81921, 11), (98304, 18),
            (98305, 9))]
    p, q, seed = 10, 2, 23
    rb = gpu.SSARaggedBatch(oversampling=p, power_iters=q, groups=[[0], [1, 2]])
    sig, W, G = rb.run([m[0] for m in mix], [m[1] for m in mix], [m[2] for m in mix], seed=seed)
    for s, (x, L, k) in enumerate(mix):
        N = len(x)
        K = N - L + 1
        Om = oracle.device_gaussian(oracle.series_seed(seed, s), K, min(k + p, L, K))
        d = oracle.decompose_randomized(x, L, k, p, Om, q=q)
        check_sigma(sig[s], d.sigma)
        for gi, g in enumerate(([0], [1, 2])):
            assert rel_l2(G[s][gi], oracle.reconstruct(d, g, N, L)) <= rec_tol(d.sigma, g), (s, N, g)
        assert np.max(np.abs(np.diag(W[s]) - 1.0)) < 1e-6
        Wr = oracle.wcorr_matrix(d, N, L)
        blk = [i for i in range(min(6, len(d.sigma)))
               if min(abs(d.sigma[i] - d.sigma[j]) / d.sigma[i] for j in range(len(d.sigma)) if j != i) > 1e-2]
        if blk:
            assert np.max(np.abs(W[s][np.ix_(blk, blk)] - Wr[np.ix_(blk, blk)])) < 1e-4, (s, N)
