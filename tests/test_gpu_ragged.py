"""Uneven batches (ssa_rbatch_*) against the FP64 oracle, against the uniform batch, and alone
versus in a mix.

Tolerances as in the single-series parity tests: singular values relative <= 1e-5 where the
relative gap to the neighbours exceeds 1e-3 (1e-4 otherwise); group reconstructions relative L2
<= 1e-5 for groups separated by a relative gap > 1e-2, else max(1e-5, 40 * 2^-24 / gap);
W-correlation diagonal 1 within 1e-6 and max abs <= 1e-4 on the leading well-separated block.
A series run alone and in a mix differs only in how its FP64 Gram partials are chunked, so the
two agree to the same tolerances.
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


def leading_block(sigma, kmax=6):
    """Leading components whose relative gap to every other computed one exceeds 1e-2."""
    return [i for i in range(min(kmax, len(sigma))) if group_gap(sigma, [i]) > 1e-2]


def test_uneven_batch_vs_oracle(gpu, oracle):
    mix = oracle.config3_batch(10, seed=2, nmin=500, nmax=20000)
    # both reconstruction paths: a series above 16384 (one FFT buffer) and small ones
    rng = np.random.default_rng(77)
    mix.append((oracle.walk_sines(rng, 18000), 4500, 12))
    mix.append((oracle.walk_sines(rng, 700), 175, 40))
    p, q, seed = 10, 2, 31
    rb = gpu.SSARaggedBatch(oversampling=p, power_iters=q, groups=[[0], [1, 2]])
    xs = [m[0] for m in mix]
    Ls = [m[1] for m in mix]
    ks = [m[2] for m in mix]
    sig, W, G = rb.run(xs, Ls, ks, seed=seed)
    for s, (x, L, k) in enumerate(mix):
        N = len(x)
        K = N - L + 1
        kp = min(k + p, L, K)
        Om = oracle.device_gaussian(oracle.series_seed(seed, s), K, kp)
        d = oracle.decompose_randomized(x, L, k, p, Om, q=q)
        check_sigma(sig[s], d.sigma)
        for gi, g in enumerate(([0], [1, 2])):
            e = rel_l2(G[s][gi], oracle.reconstruct(d, g, N, L))
            assert e <= rec_tol(d.sigma, g), (s, N, g, e)
        Wr = oracle.wcorr_matrix(d, N, L)
        assert np.max(np.abs(np.diag(W[s]) - 1.0)) < 1e-6
        blk = leading_block(d.sigma)
        if blk:
            assert np.max(np.abs(W[s][np.ix_(blk, blk)] - Wr[np.ix_(blk, blk)])) < 1e-4, (s, N)


def test_uneven_equals_uniform_for_equal_shapes(gpu, oracle):
    B, N, L, k = 6, 3000, 750, 20
    X = oracle.config2_batch(B, seed=5, N=N)
    ub = gpu.SSABatch(B, N, L, k, oversampling=10, power_iters=2)
    s_u, W_u, G_u = ub.run(X, seed=9)
    rb = gpu.SSARaggedBatch(oversampling=10, power_iters=2)
    s_r, W_r, G_r = rb.run(list(X), [L] * B, [k] * B, seed=9)
    for s in range(B):
        np.testing.assert_allclose(s_r[s], s_u[s], rtol=1e-12, atol=0)
        np.testing.assert_allclose(G_r[s], G_u[s], rtol=0, atol=1e-9 * np.abs(G_u[s]).max())
        np.testing.assert_allclose(W_r[s], W_u[s], rtol=0, atol=1e-9)


def test_alone_equals_in_mix(gpu, oracle):
    mix = oracle.config3_batch(8, seed=12, nmin=500, nmax=9000)
    xs = [m[0] for m in mix]
    Ls = [m[1] for m in mix]
    ks = [m[2] for m in mix]
    rb = gpu.SSARaggedBatch(oversampling=10, power_iters=2)
    sig, W, G = rb.run(xs, Ls, ks, seed=4)
    for s in (0, 3, 7):
        # the same series at the same batch position (its generator seed depends on it), the
        # positions before it taken by short noise series in another FFT-length bucket
        pad_x = [np.random.default_rng(i).standard_normal(64) for i in range(s)] + [xs[s]]
        pad_L = [16] * s + [Ls[s]]
        pad_k = [2] * s + [ks[s]]
        s1, W1, G1 = rb.run(pad_x, pad_L, pad_k, seed=4)
        check_sigma(s1[s], sig[s])
        for gi, g in enumerate(([0], [1, 2])):
            assert rel_l2(G1[s][gi], G[s][gi]) <= rec_tol(sig[s], g)


def test_serialized_profiling_is_bit_identical(gpu, oracle):
    """Profiling mode 2 only chains the FFT-length buckets on the streams: the same kernels on the
    same data, so the outputs are bit-identical and every kernel kind reports launches."""
    mix = oracle.config3_batch(12, seed=21, nmin=500, nmax=70000)
    xs, Ls, ks = [m[0] for m in mix], [m[1] for m in mix], [m[2] for m in mix]
    rb = gpu.SSARaggedBatch(oversampling=10, power_iters=2)
    ref = rb.run(xs, Ls, ks, seed=8)
    for serialize in (False, True):
        rb.set_profiling(True, serialize=serialize)
        rb.profile()
        out = rb.run(xs, Ls, ks, seed=8)
        prof = rb.profile()
        rb.set_profiling(False)
        for a, b in zip(out, ref):
            for s in range(len(xs)):
                assert np.array_equal(a[s], b[s]), s
        assert prof["corr"][1] > 0 and prof["corr"][0] > 0
    assert gpu._lib.ssa_rbatch_set_profiling(rb._h, 3) == -1  # unknown mode


def test_per_series_outputs_mask(gpu, oracle):
    """want_w: series without W compute only the elementary reconstructions their groups use.
    The decomposition and the group sums do not depend on the mask (bit-identical); flagged
    series get the same W as in the plain run, the others a zero W block."""
    mix = oracle.config3_batch(14, seed=31, nmin=500, nmax=70000)
    xs, Ls, ks = [m[0] for m in mix], [m[1] for m in mix], [m[2] for m in mix]
    want = np.arange(len(xs)) % 3 == 0
    rb = gpu.SSARaggedBatch(oversampling=10, power_iters=2)
    s0, W0, G0 = rb.run(xs, Ls, ks, seed=6)
    s1, W1, G1 = rb.run(xs, Ls, ks, seed=6, want_w=want)
    for i in range(len(xs)):
        assert np.array_equal(s0[i], s1[i]) and np.array_equal(G0[i], G1[i]), i
        if want[i]:
            assert np.array_equal(W0[i], W1[i]), i
        else:
            assert not W1[i].any(), i
    s2, W2, G2 = rb.run(xs, Ls, ks, seed=6)  # a plain run after a masked one is whole again
    for i in range(len(xs)):
        assert np.array_equal(W0[i], W2[i]) and np.array_equal(G0[i], G2[i]), i
    with pytest.raises(ValueError):
        rb.run(xs, Ls, ks, want_w=want[:-1])


def test_uneven_batch_rejects_bad_series(gpu, oracle):
    rb = gpu.SSARaggedBatch()
    x = np.sin(np.arange(100.0)) + 0.1 * np.random.default_rng(1).standard_normal(100)
    with pytest.raises(RuntimeError):
        rb.run([x], [100], [5])  # L > N - 1
    with pytest.raises(RuntimeError):
        rb.run([np.zeros(140000)], [100], [5])  # beyond the largest FFT length
    s, W, G = rb.run([x, x[:50]], [25, 10], [4, 3])  # still usable afterwards
    assert len(s[0]) == 4 and len(s[1]) == 3


def test_single_series_wcorr_one_buffer_path(gpu, oracle):
    """N = 20000 needs the one-buffer elementary reconstruction (FFT length 32768)."""
    rng = np.random.default_rng(8)
    x = oracle.walk_sines(rng, 20000)
    N, L, k, p = 20000, 5000, 10, 10
    K = N - L + 1
    Om = rng.standard_normal((K, k + p))
    d = oracle.decompose_randomized(x, L, k, p, Om, q=2)
    s = gpu.SSA(x, L)
    s.decompose(k, oversampling=p, power_iters=2, omega=Om)
    check_sigma(s.singular_values, d.sigma)
    W = s.wcorr_matrix()
    Wr = oracle.wcorr_matrix(d, N, L)
    assert np.max(np.abs(np.diag(W) - 1.0)) < 1e-6
    blk = leading_block(d.sigma)
    assert blk and np.max(np.abs(W[np.ix_(blk, blk)] - Wr[np.ix_(blk, blk)])) < 1e-4


def test_multi_length_sweeps_equal_per_length_buckets(gpu, oracle):
    """Series of real FFT lengths 512 .. 16384 share one persistent, queue-fed sweep launch (tiles
    of one series, column group and length; several columns of a short length side by side in a
    CTA). Each column runs the same transform code as the one-length kernel; only the FP64 Gram
    chunking changes with the bucket sizes, so the results agree to the parity tolerances, and
    both agree with the oracle."""
    rng = np.random.default_rng(41)
    Ns = [300, 600, 1000, 1900, 2100, 4000, 4500, 7000, 9000, 15000, 16384, 20000]
    xs = [oracle.walk_sines(rng, N) for N in Ns]
    Ls = [N // 4 for N in Ns]
    ks = [int(k) for k in rng.integers(8, 40, len(Ns))]
    rb = gpu.SSARaggedBatch(oversampling=10, power_iters=2)
    assert gpu.multi_length()
    try:
        s_m, W_m, G_m = rb.run(xs, Ls, ks, seed=5)
        gpu.set_multi_length(False)
        s_p, W_p, G_p = rb.run(xs, Ls, ks, seed=5)
    finally:
        gpu.set_multi_length(True)
    for i in range(len(Ns)):
        check_sigma(s_m[i], s_p[i])
        for gi, g in enumerate(([0], [1, 2])):
            assert rel_l2(G_m[i][gi], G_p[i][gi]) <= rec_tol(s_p[i], g), (Ns[i], g)
        N, L, k = Ns[i], Ls[i], ks[i]
        K = N - L + 1
        kk, kp = oracle.clamp_kp(L, K, k, 10)
        d = oracle.decompose_randomized(xs[i], L, kk, 10, oracle.device_gaussian(oracle.series_seed(5, i), K, kp), q=2)
        check_sigma(s_m[i], d.sigma)
        for gi, g in enumerate(([0], [1, 2])):
            assert rel_l2(G_m[i][gi], oracle.reconstruct(d, g, N, L)) <= rec_tol(d.sigma, g)


def test_graph_replays_equal_direct_runs(gpu, oracle):
    """A run with the previous run's launch signature is captured as a CUDA graph and later runs
    replay it (job tables restored, the generator seed read from device memory): the outputs are
    bit-identical to direct launches with graphs off, for every seed."""
    mix = oracle.config3_batch(10, seed=33, nmin=500, nmax=40000)
    xs, Ls, ks = [m[0] for m in mix], [m[1] for m in mix], [m[2] for m in mix]
    seeds = [11, 12, 13, 14]
    g = gpu.SSARaggedBatch(oversampling=10, power_iters=2)
    outs = [g.run(xs, Ls, ks, seed=sd) for sd in seeds]
    st = g.graph_stats()
    assert st == {"captures": 1, "replays": 2}, st
    d = gpu.SSARaggedBatch(oversampling=10, power_iters=2)
    d.set_graphs(False)
    for sd, out in zip(seeds, outs):
        ref = d.run(xs, Ls, ks, seed=sd)
        for a, b in zip(out, ref):
            for s in range(len(xs)):
                assert np.array_equal(a[s], b[s]), (sd, s)
    assert d.graph_stats() == {"captures": 0, "replays": 0}
    # a different shape list is a new signature: direct launch, no replay of the old graph
    g.run(xs[:5], Ls[:5], ks[:5], seed=1)
    assert g.graph_stats()["replays"] == 2


def test_cluster32k_form_equals_single_cta_form(gpu, oracle):
    """Real FFT length 32768 on 2-CTA clusters (8192 points per CTA, exchange through distributed
    shared memory) or on one 1024-thread CTA: the uneven batch (sweeps, spectra, elementary
    reconstructions, W) and the single-series API (cached-spectra reconstruction) agree with each
    other and with the oracle."""
    import ctypes

    lib = gpu._lib
    lib.ssa_b200_set_cluster32k.argtypes = [ctypes.c_int]
    lib.ssa_b200_cluster32k.restype = ctypes.c_int
    rng = np.random.default_rng(51)
    Ns = [16500, 20000, 24000, 30000, 32768]
    xs = [oracle.walk_sines(rng, N) for N in Ns]
    Ls = [N // 4 for N in Ns]
    ks = [12, 20, 30, 16, 25]
    rb = gpu.SSARaggedBatch(oversampling=10, power_iters=2)
    assert lib.ssa_b200_cluster32k() == 0
    outs = {}
    try:
        for on in (0, 1):
            lib.ssa_b200_set_cluster32k(on)
            outs[on] = rb.run(xs, Ls, ks, seed=6)
            s = gpu.SSA(xs[1], Ls[1])
            s.decompose(20, oversampling=10, power_iters=2)
            outs[on] = outs[on] + (s.reconstruct([1, 2]), s.wcorr_matrix())
    finally:
        lib.ssa_b200_set_cluster32k(0)
    (s0, W0, G0, r0, w0), (s1, W1, G1, r1, w1) = outs[0], outs[1]
    for i in range(len(Ns)):
        check_sigma(s1[i], s0[i])
        for gi, g in enumerate(([0], [1, 2])):
            assert rel_l2(G1[i][gi], G0[i][gi]) <= rec_tol(s0[i], g)
        blk = leading_block(s0[i])
        assert np.max(np.abs(W1[i][np.ix_(blk, blk)] - W0[i][np.ix_(blk, blk)])) < 1e-4
        N, L, k = Ns[i], Ls[i], ks[i]
        K = N - L + 1
        kk, kp = oracle.clamp_kp(L, K, k, 10)
        d = oracle.decompose_randomized(xs[i], L, kk, 10, oracle.device_gaussian(oracle.series_seed(6, i), K, kp), q=2)
        check_sigma(s1[i], d.sigma)
        for gi, g in enumerate(([0], [1, 2])):
            assert rel_l2(G1[i][gi], oracle.reconstruct(d, g, N, L)) <= rec_tol(d.sigma, g)
    assert rel_l2(r1, r0) <= 1e-5 and np.max(np.abs(w1[:3, :3] - w0[:3, :3])) < 1e-4
