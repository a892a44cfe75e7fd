"""MSSA (MKL/ssa_opt.h:3880-4283) and Cadzow iterations (:3165-3442) on the GPU against the
FP64 oracle, through the C ABI of libssa.so.

Tolerances follow the single-series parity tests: singular values relative <= 1e-5 where the
relative gap to the neighbours exceeds 1e-3 (1e-4 otherwise); reconstructions relative L2
<= 1e-5 for groups separated by a relative gap > 1e-2, max(1e-5, 40 * 2^-24 / gap) otherwise.
Cadzow repeats decompose + reconstruct, so its signals are held to CADZOW_TOL = 1e-4 relative
L2 after up to 6 iterations, and its reported relative differences to 1e-5 absolute.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIG_TOL = 1e-5
REC_TOL = 1e-5
CADZOW_TOL = 1e-4


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


def mssa_case(oracle, seed=4, Mch=4, N=2000):
    rng = np.random.default_rng(seed)
    return oracle.config4_instance(rng, Mch=Mch, N=N), rng


# ---- MSSA ----------------------------------------------------------------------------------


@pytest.mark.parametrize("q", [0, 2])
def test_mssa_parity_host_omega(gpu, oracle, q):
    X, rng = mssa_case(oracle)
    Mch, N = X.shape
    L, k, p = 500, 12, 8
    K = N - L + 1
    Om = rng.standard_normal((K, k + p))
    d = oracle.mssa_decompose(X, L, k, p, Om, q=q)
    m = gpu.MSSA(X, L)
    m.decompose(k, oversampling=p, power_iters=q, omega=Om)
    U, V, s = m.factors()
    assert U.shape == (Mch * L, k) and V.shape == (K, k)
    check_sigma(s, d.sigma)
    assert np.max(np.abs(U.T @ U - np.eye(k))) < 1e-4
    assert np.max(np.abs(V.T @ V - np.eye(k))) < 1e-4
    assert np.all(U.sum(axis=0) >= 0)  # sign rule over all M L rows (:4195-4205)
    for ch in (0, Mch - 1):
        for g in ([0], [1, 2]):
            e = rel_l2(m.reconstruct(ch, g), oracle.mssa_reconstruct(d, ch, g, Mch, N, L))
            assert e <= rec_tol(d.sigma, g), (ch, g, e)
    c = m.series_contributions()
    cr = oracle.mssa_series_contributions(d, Mch, L)
    assert np.max(np.abs(c.sum(axis=0) - 1.0)) < 1e-5
    sep = [i for i in range(k) if group_gap(d.sigma, [i]) > 1e-2]
    assert np.max(np.abs(c[:, sep] - cr[:, sep])) < 1e-4
    ve = m.variance_explained(0, 3)
    assert abs(ve - d.eigenvalues[:4].sum() / d.total_variance) < 1e-6


def test_mssa_config4_full_size(gpu, oracle):
    """One instance at the full MSSA workload shape (M = 16 channels, N = 20000, L = 5000, k = 50,
    p = 10, q = 2, host test matrix), then 10 rank-50 Cadzow iterations on a channel, against the
    oracle; same tolerances as above."""
    rng = np.random.default_rng(3)
    X = oracle.config4_instance(rng, Mch=16, N=20000)
    Mch, N = X.shape
    L, k, p = 5000, 50, 10
    K = N - L + 1
    Om = rng.standard_normal((K, k + p))
    d = oracle.mssa_decompose(X, L, k, p, Om, q=2)
    m = gpu.MSSA(X, L)
    m.decompose(k, oversampling=p, power_iters=2, omega=Om)
    check_sigma(m.singular_values, d.sigma)
    for ch in (0, Mch - 1):
        for g in ([0], [1, 2]):
            e = rel_l2(m.reconstruct(ch, g), oracle.mssa_reconstruct(d, ch, g, Mch, N, L))
            assert e <= rec_tol(d.sigma, g), (ch, g, e)
    x = X[0]
    rank, iters = 50, 10
    Omc = oracle.device_gaussian(oracle.single_series_seed(0), K, rank + 8)
    y_ref, it_ref, diff_ref, _ = oracle.cadzow(x, L, rank, iters, 1e-14, Omc)
    r = gpu.cadzow(x, L, rank, max_iter=iters, tol=1e-14)
    assert r.iterations == it_ref == iters
    assert rel_l2(r.signal, y_ref) <= CADZOW_TOL
    assert abs(r.final_diff - diff_ref) <= 1e-5


def test_mssa_default_generator_matches_replica(gpu, oracle):
    X, _ = mssa_case(oracle, seed=5, Mch=3, N=1200)
    Mch, N = X.shape
    L, k = 300, 8
    K = N - L + 1
    m = gpu.MSSA(X, L)
    m.decompose(k)  # p = 8, q = 0, first generated matrix of the context
    Om = oracle.device_gaussian(oracle.mssa_seed(0), K, k + 8)
    d = oracle.mssa_decompose(X, L, k, 8, Om, q=0)
    check_sigma(m.singular_values, d.sigma)
    assert rel_l2(m.reconstruct(1, [0]), oracle.mssa_reconstruct(d, 1, [0], Mch, N, L)) <= rec_tol(d.sigma, [0])


def test_mssa_single_channel_is_ssa(gpu, oracle):
    x, _, _ = oracle.config1(seed=3)
    N, L, k, p = 1000, 250, 10, 10
    K = N - L + 1
    Om = np.random.default_rng(9).standard_normal((K, k + p))
    m = gpu.MSSA(x[None, :], L)
    m.decompose(k, oversampling=p, power_iters=1, omega=Om)
    s = gpu.SSA(x, L)
    s.decompose(k, oversampling=p, power_iters=1, omega=Om)
    assert np.max(np.abs(m.singular_values - s.singular_values) / s.singular_values) < 1e-5
    d = oracle.decompose_randomized(x, L, k, p, Om, q=1)
    assert rel_l2(m.reconstruct(0, [0]), oracle.reconstruct(d, [0], N, L)) <= rec_tol(d.sigma, [0])


def test_mssa_reconstruct_all_and_errors(gpu, oracle):
    X, _ = mssa_case(oracle, seed=6, Mch=3, N=900)
    Mch, N = X.shape
    L = 200
    m = gpu.MSSA(X, L)
    with pytest.raises(RuntimeError):
        m.reconstruct(0, [0])
    m.decompose(6)
    R = m.reconstruct_all([0, 1, 2])
    for ch in range(Mch):
        assert np.array_equal(R[ch], m.reconstruct(ch, [0, 1, 2]))
    with pytest.raises(RuntimeError):
        m.reconstruct(Mch, [0])
    full = m.reconstruct_all(list(range(m.n_components)))
    assert rel_l2(full, X) < 0.7  # six leading components carry most of the energy (SNR 5 dB)
    with pytest.raises(ValueError):
        gpu.MSSA(X, N)  # L > N - 1


# ---- Cadzow --------------------------------------------------------------------------------


def two_sines(N, noise, seed):
    rng = np.random.default_rng(seed)
    t = np.arange(N)
    clean = np.sin(2 * np.pi * t / 17) + 0.6 * np.sin(2 * np.pi * t / 7.3 + 1.0)
    return clean + noise * rng.standard_normal(N), clean


def test_cadzow_randomized_branch(gpu, oracle):
    x, clean = two_sines(1000, 0.3, 1)
    N, L, rank, iters = 1000, 250, 4, 6
    K = N - L + 1
    assert rank + 8 < min(L, K) // 2
    Om = oracle.device_gaussian(oracle.single_series_seed(0), K, rank + 8)
    y_ref, it_ref, diff_ref, conv_ref = oracle.cadzow(x, L, rank, iters, 1e-14, Om)
    r = gpu.cadzow(x, L, rank, max_iter=iters, tol=1e-14)
    assert r.iterations == it_ref == iters and not r.converged
    assert rel_l2(r.signal, y_ref) <= CADZOW_TOL
    assert abs(r.final_diff - diff_ref) <= 1e-5
    assert rel_l2(r.signal, clean) < rel_l2(x, clean)  # denoises


def test_cadzow_block_branch(gpu, oracle):
    x, _ = two_sines(100, 0.05, 2)
    N, L, rank, iters = 100, 24, 4, 4
    K = N - L + 1
    assert not rank + 8 < min(L, K) // 2
    V0 = oracle.device_gaussian(oracle.series_seed(oracle.block_seed(0), 0), K, rank)
    y_ref, it_ref, diff_ref, _ = oracle.cadzow(x, L, rank, iters, 1e-14, V0)
    r = gpu.cadzow(x, L, rank, max_iter=iters, tol=1e-14)
    assert r.iterations == it_ref
    assert rel_l2(r.signal, y_ref) <= CADZOW_TOL
    assert abs(r.final_diff - diff_ref) <= 1e-5


def test_cadzow_converges_and_weighted(gpu, oracle):
    x, _ = two_sines(800, 0.02, 3)
    N, L, rank = 800, 200, 4
    K = N - L + 1
    Om = oracle.device_gaussian(oracle.single_series_seed(0), K, rank + 8)
    y_ref, it_ref, diff_ref, conv_ref = oracle.cadzow(x, L, rank, 50, 1e-3, Om)
    r = gpu.cadzow(x, L, rank, max_iter=50, tol=1e-3)
    assert conv_ref and r.converged and r.final_diff < 1e-3
    assert abs(r.iterations - it_ref) <= 1
    assert rel_l2(r.signal, y_ref) <= CADZOW_TOL
    yw_ref, *_ = oracle.cadzow_weighted(x, L, rank, 3, 1e-14, 0.25, Om)
    w = gpu.cadzow(x, L, rank, max_iter=3, tol=1e-14, alpha=0.25)
    assert rel_l2(w.signal, yw_ref) <= CADZOW_TOL
    for bad in (0.0, 1.5):
        with pytest.raises(RuntimeError):
            gpu.cadzow(x, L, rank, max_iter=3, alpha=bad)
    with pytest.raises(RuntimeError):
        gpu.cadzow(x, L, 0, max_iter=3)
    with pytest.raises(RuntimeError):
        gpu.cadzow(x, L, rank, max_iter=0)


def test_cadzow_inplace(gpu, oracle):
    x, _ = two_sines(600, 0.2, 4)
    N, L, rank, iters = 600, 150, 4, 5
    K = N - L + 1
    s = gpu.SSA(x, L)
    s.prepare(rank, 8)
    oms = [oracle.device_gaussian(oracle.single_series_seed(i), K, rank + 8) for i in range(iters)]
    y_ref, it_ref, diff_ref, conv_ref, _ = oracle.cadzow_inplace(x, L, rank, iters, 1e-14, oms)
    r = s.cadzow_inplace(rank, max_iter=iters, tol=1e-14)
    assert r.iterations == it_ref == iters
    assert rel_l2(r.signal, y_ref) <= CADZOW_TOL
    assert abs(r.final_diff - diff_ref) <= 1e-5
    assert s.n_components == rank
    # the context stays usable: a fresh decomposition of its (updated) signal works
    s.decompose(rank, oversampling=8)
    assert len(s.singular_values) == rank


def _mbatch_check(gpu, oracle, I, M, N, L, k, iters, seed, check=None):
    rng = np.random.default_rng(seed)
    X = np.stack([oracle.config4_instance(rng, Mch=M, N=N) for _ in range(I)])
    mb = gpu.SSAMultiBatch(I, M, N, L, k, oversampling=10, power_iters=2)
    out, sig, diff = mb.run(X, iters, seed=seed)
    K = N - L + 1
    for i in (range(I) if check is None else check):
        Om = oracle.device_gaussian(oracle.series_seed(seed, i), K, mb.kp)
        y_ref, s_ref, d_ref = oracle.mssa_cadzow(X[i], L, mb.k, iters, 10, Om, q=2)
        lead = min(5, mb.k)
        assert np.max(np.abs(sig[i][:lead] - s_ref[:lead]) / s_ref[:lead]) <= 1e-5, i
        assert rel_l2(out[i], y_ref) <= CADZOW_TOL, (i, rel_l2(out[i], y_ref))
        assert np.max(np.abs(diff[i] - d_ref)) <= 1e-5, (i, diff[i], d_ref)
    return out, diff


def test_multichannel_batch_cadzow_vs_oracle(gpu, oracle):
    """Batched multichannel SSA with Cadzow iterations (ssa_mbatch): three instances of four
    channels, block power of each stacked operator (one block of kp columns, two subspace
    iterations, generated start block per instance), three multivariate Cadzow iterations; every
    instance against the oracle's restatement with the same start block."""
    out, diff = _mbatch_check(gpu, oracle, I=3, M=4, N=3000, L=750, k=12, iters=3, seed=21)
    assert np.all(diff[:, -1] < diff[:, 0])  # the iteration contracts


def _oracle_instance(args):
    import ssa_oracle

    x, L, k, iters, Om = args
    return ssa_oracle.mssa_cadzow(x, L, k, iters, 10, Om, q=2)


def test_multichannel_batch_full_shape(gpu, oracle):
    """The multichannel workload's shape (16 channels of N = 20000, L = 5000, rank 50): four
    instances in one batch, two Cadzow iterations, every instance against the oracle (computed in
    four spawned processes)."""
    import multiprocessing as mp
    import os

    I, M, N, L, k, iters, seed = 4, 16, 20000, 5000, 50, 2, 3
    rng = np.random.default_rng(seed)
    X = np.stack([oracle.config4_instance(rng, Mch=M, N=N) for _ in range(I)])
    mb = gpu.SSAMultiBatch(I, M, N, L, k, oversampling=10, power_iters=2)
    out, sig, diff = mb.run(X, iters, seed=seed)
    K = N - L + 1
    jobs = [(X[i], L, mb.k, iters, oracle.device_gaussian(oracle.series_seed(seed, i), K, mb.kp)) for i in range(I)]
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "4")
    with mp.get_context("spawn").Pool(I) as pool:
        refs = pool.map(_oracle_instance, jobs)
    lead = min(5, mb.k)
    for i, (y_ref, s_ref, d_ref) in enumerate(refs):
        assert np.max(np.abs(sig[i][:lead] - s_ref[:lead]) / s_ref[:lead]) <= 1e-5, i
        assert rel_l2(out[i], y_ref) <= CADZOW_TOL, (i, rel_l2(out[i], y_ref))
        assert np.max(np.abs(diff[i] - d_ref)) <= 1e-5, (i, diff[i], d_ref)
