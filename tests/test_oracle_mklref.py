"""Pins the NumPy oracle to the reference's own product path, MKL/ssa_opt.h.

The unmodified header is compiled by oracle/Makefile against the MKL-compatibility shim
(oracle/mklshim/: own DFTI FFT, VML loops, VSL draws from a registered buffer, CBLAS/LAPACKE from
scipy's OpenBLAS) into oracle/_ref/libssa_mklshim.so. Every case registers the test matrix (or
uniform start blocks) that the reference's RNG stream would draw, runs the reference's call
sequence, and compares with the oracle given the same draws. Tolerances are FP64 rounding-level:
both sides run the same algorithm with the same LAPACK routines (the FFTs differ: the shim's own
radix-4 Stockham against numpy's pocketfft).
"""
import numpy as np
import pytest


def _cfg3_series(oracle, n=5, seed=2):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = int(round(np.exp(rng.uniform(np.log(500), np.log(6000)))))
        L = max(2, int(round(N / 4)))
        k = int(rng.integers(10, 51))
        x = oracle.walk_sines(rng, N)
        out.append((x, L, k))
    return out


def _align(A, B):
    """Columns of B flipped to the sign of A's (both follow the reference's sign rule; this only
    guards components whose column sum is ~0)."""
    s = np.sign(np.sum(A * B, axis=0))
    s[s == 0] = 1.0
    return B * s


def _check_dec(sig, U, V, d, rtol=1e-10):
    assert sig.shape == d.sigma.shape
    rel = np.abs(sig - d.sigma) / d.sigma
    assert rel.max() < rtol, rel.max()
    # vectors: rounding-level for separated values; a pair with a relative gap g may rotate by
    # ~eps/g inside its plane
    gaps = np.full(len(sig), np.inf)
    gaps[:-1] = np.minimum(gaps[:-1], (sig[:-1] - sig[1:]) / sig[0])
    gaps[1:] = np.minimum(gaps[1:], (sig[:-1] - sig[1:]) / sig[0])
    sep = gaps > 1e-6
    Ua = _align(d.U, U)
    Va = _align(d.V, V)
    assert np.max(np.abs(Ua[:, sep] - d.U[:, sep])) < 1e-8
    assert np.max(np.abs(Va[:, sep] - d.V[:, sep])) < 1e-8


def test_mklref_matvec_kats(oracle, mklref):
    """MKL/test/ssa_opt_test.c:1464-1559 (FFT matvec / adjoint vs direct sums, < 1e-10) run on the
    reference's own ssa_opt_hankel_matvec / _T, and the oracle's FFT matvec against them."""
    N, L = 100, 25
    K = N - L + 1
    i = np.arange(N)
    x = np.sin(0.1 * i) + 0.5 * np.cos(0.25 * i)
    v = np.cos(0.05 * np.arange(K))
    u = np.cos(0.07 * np.arange(L))
    y, z = np.zeros(L), np.zeros(K)
    assert mklref.lib.mkr_matvec(mklref.d(x), N, L, mklref.d(v), mklref.d(y), 0) == 0
    assert mklref.lib.mkr_matvec(mklref.d(x), N, L, mklref.d(u), mklref.d(z), 1) == 0
    assert np.max(np.abs(y - oracle.hankel_matvec_direct(x, v, L))) < 1e-10
    assert np.max(np.abs(z - oracle.hankel_matvec_T_direct(x, u, L))) < 1e-10
    assert np.max(np.abs(y - oracle.hankel_matvec(x, v, L))) < 1e-12
    assert np.max(np.abs(z - oracle.hankel_matvec_T(x, u, L))) < 1e-12


@pytest.mark.parametrize("N,L", [(4, 2), (5, 4), (777, 300), (4096, 1024), (20000, 5000)])
def test_mklref_fft_lengths_and_matvec(oracle, mklref, N, L):
    """FFT length next_pow2(N + K - 1) and the matvecs at odd and large shapes."""
    rng = np.random.default_rng(N)
    x = rng.standard_normal(N)
    K = N - L + 1
    fl, bs = np.zeros(1, dtype=np.int32), np.zeros(1, dtype=np.int32)
    assert mklref.lib.mkr_dims(mklref.d(x), N, L, mklref.i(fl), mklref.i(bs)) == 0
    assert fl[0] == oracle.ref_fft_len(N, L)
    v, u = rng.standard_normal(K), rng.standard_normal(L)
    y, z = np.zeros(L), np.zeros(K)
    mklref.lib.mkr_matvec(mklref.d(x), N, L, mklref.d(v), mklref.d(y), 0)
    mklref.lib.mkr_matvec(mklref.d(x), N, L, mklref.d(u), mklref.d(z), 1)
    sc = np.linalg.norm(x)
    assert np.max(np.abs(y - oracle.hankel_matvec_direct(x, v, L))) < 1e-12 * sc * np.linalg.norm(v)
    assert np.max(np.abs(z - oracle.hankel_matvec_T_direct(x, u, L))) < 1e-12 * sc * np.linalg.norm(u)


def test_mklref_randomized_config1(oracle, mklref):
    """ssa_opt_decompose_randomized (MKL/ssa_opt.h:1685-1763) at the single-series workload
    (N = 1000, L = 250, k = 50, p = 10) with the workload's Gaussian test matrix: the oracle's
    randomized restatement at q = 0 equals it to FP64 rounding."""
    x, _, Om = oracle.config1(seed=0, N=1000, L=250, k=50, p=10)
    sig, U, V, tv = mklref.randomized(x, 250, 50, 10, Om)
    d = oracle.decompose_randomized(x, 250, 50, 10, Om, q=0)
    _check_dec(sig, U, V, d)
    assert abs(tv - d.total_variance) < 1e-10 * d.total_variance
    # the reference's U is orthonormal (its pure-C sibling's is not)
    assert np.max(np.abs(U.T @ U - np.eye(U.shape[1]))) < 1e-12


def test_mklref_randomized_uneven_series(oracle, mklref):
    """Five series of the uneven-batch generator (random walk + sinusoids + noise), each with its
    own k and a Gaussian test matrix."""
    rng = np.random.default_rng(77)
    for x, L, k in _cfg3_series(oracle):
        N = len(x)
        K = N - L + 1
        kk, kp = oracle.clamp_kp(L, K, k, 10)
        Om = oracle.gaussian_omega(rng, K, kp)
        sig, U, V, _ = mklref.randomized(x, L, k, 10, Om)
        _check_dec(sig, U, V, oracle.decompose_randomized(x, L, k, 10, Om, q=0))


def test_mklref_pipeline(oracle, mklref):
    """Reconstruction (uncached, MKL/ssa_opt.h:2325-2400), W-correlation slow and cached/DSYRK
    paths (:2407-2548), LRF (:2766-2816) and R-forecast (:2843-2867) after the reference's own
    decomposition, against the oracle on the same factors."""
    N, L, k, p = 1000, 250, 20, 10
    x, _, Om = oracle.config1(seed=3, N=N, L=L, k=k, p=p)
    mklref.set_gaussian(mklref.omega_draws(Om))
    d = oracle.decompose_randomized(x, L, k, p, Om, q=0)
    groups = np.array([0, 1, 2, 3, 4, 5], dtype=np.int32)
    sizes = np.array([1, 2, 3], dtype=np.int32)
    rec = np.zeros(3 * N)
    fg = np.array([0, 1, 2], dtype=np.int32)
    h = 50
    for w_mode in (1, 2):
        W = np.zeros(k * k)
        fc = np.zeros(h)
        R = np.zeros(L - 1)
        vert = np.zeros(1)
        sig = np.zeros(k)
        n = mklref.lib.mkr_pipeline(mklref.d(x), N, L, k, p, mklref.i(groups), mklref.i(sizes), 3,
                                    mklref.d(rec), w_mode, mklref.d(W), mklref.i(fg), 3, h, mklref.d(fc),
                                    mklref.d(R), mklref.d(vert), mklref.d(sig))
        assert n == k
        assert np.max(np.abs(sig - d.sigma) / d.sigma) < 1e-10
        for g, grp in enumerate(([0], [1, 2], [3, 4, 5])):
            ref = oracle.reconstruct(d, grp, N, L)
            assert np.max(np.abs(rec[g * N:(g + 1) * N] - ref)) < 1e-9 * np.max(np.abs(ref))
        Wo = oracle.wcorr_matrix(d, N, L)
        assert np.max(np.abs(W.reshape(k, k) - Wo)) < 1e-9
        Ro, vo = oracle.compute_lrf(d, [0, 1, 2], L)
        assert abs(vert[0] - vo) < 1e-12
        assert np.max(np.abs(R - Ro)) < 1e-9 * max(1.0, np.max(np.abs(Ro)))
        fo = oracle.forecast(d, [0, 1, 2], h, N, L)
        assert np.max(np.abs(fc - fo)) < 1e-8 * max(1.0, np.max(np.abs(fo)))


@pytest.mark.parametrize("iters", [3, 12, 40])
def test_mklref_block_power(oracle, mklref, iters):
    """ssa_opt_decompose_block (MKL/ssa_opt.h:1765-1933) with registered uniform start blocks:
    the oracle's block restatement given the same blocks. An unconverged block iteration over
    nearly equal singular values (here pairs 1316/1309 and 174.8/174.1) amplifies rounding: the
    bar at 12 and 40 iterations is ten times the oracle's own change when its start blocks move by
    1e-13 relative (measured here), at 3 iterations FP64 rounding."""
    N, L, k, b = 600, 150, 9, 4
    x = oracle.reference_test_signal(N)
    K = N - L + 1
    u = np.random.default_rng(5).random(K * k)
    mklref.set_uniform(u)
    sig, U, V = np.zeros(k), np.zeros(L * k), np.zeros(K * k)
    n = mklref.lib.mkr_block(mklref.d(x), N, L, k, b, iters, mklref.d(sig), mklref.d(U), mklref.d(V))
    mklref.set_uniform(None)
    assert n == k
    V0 = (u - 0.5).reshape(k, K).T
    d = oracle.decompose_block(x, L, k, b, iters, oracle._split_blocks(V0, k, b))
    jitter = 1.0 + 1e-13 * np.random.default_rng(1).standard_normal(V0.shape)
    d2 = oracle.decompose_block(x, L, k, b, iters, oracle._split_blocks(V0 * jitter, k, b))
    sens = np.max(np.abs(d2.sigma - d.sigma) / d.sigma)
    rel = np.max(np.abs(sig - d.sigma) / d.sigma)
    assert rel <= max(1e-12, 10 * sens), (rel, sens)
    if iters == 3:
        _check_dec(sig, U.reshape(k, L).T, V.reshape(k, K).T, d, rtol=1e-12)
    # the well-separated leading components are at rounding level in every case
    Ua = _align(d.U[:, :3], U.reshape(k, L).T[:, :3])
    assert np.max(np.abs(Ua - d.U[:, :3])) < 1e-9


def test_mklref_wcorr_consumers(oracle, mklref):
    """ssa_opt_wcorr_pair / component_stats / find_periodic_pairs (MKL/ssa_opt.h:2551-2756) on
    the reference's decomposition: the pair values equal the oracle's W entries; the statistics
    follow their definitions."""
    N, L, k, p = 1000, 250, 16, 10
    x, _, Om = oracle.config1(seed=1, N=N, L=L, k=k, p=p)
    mklref.set_gaussian(mklref.omega_draws(Om))
    d = oracle.decompose_randomized(x, L, k, p, Om, q=0)
    pi = np.array([0, 1, 1, 3, 5], dtype=np.int32)
    pj = np.array([0, 2, 3, 4, 9], dtype=np.int32)
    pv = np.zeros(5)
    gaps, cum, sd = np.zeros(k - 1), np.zeros(k), np.zeros(k)
    sug = np.zeros(1, dtype=np.int32)
    pairs = np.zeros(2 * 8, dtype=np.int32)
    npair = np.zeros(1, dtype=np.int32)
    n = mklref.lib.mkr_wcorr_consumers(mklref.d(x), N, L, k, p, mklref.i(pi), mklref.i(pj), 5, mklref.d(pv),
                                       mklref.d(gaps), mklref.d(cum), mklref.d(sd), mklref.i(sug),
                                       mklref.i(pairs), 8, 0.1, 0.5, mklref.i(npair))
    assert n == k
    W = oracle.wcorr_matrix(d, N, L)
    assert np.max(np.abs(pv - W[pi, pj])) < 1e-9
    s = d.sigma
    assert np.allclose(gaps, s[:-1] / (s[1:] + 1e-300), rtol=1e-10)
    assert sug[0] == int(np.argmax(gaps)) + 1
    lam = s * s
    assert np.allclose(cum, np.cumsum(lam) / lam.sum(), atol=1e-12)
    ls = np.log(s + 1e-300)
    assert sd[0] == 0.0 and sd[-1] == 0.0
    assert np.allclose(sd[1:-1], ls[:-2] - 2 * ls[1:-1] + ls[2:], atol=1e-10)
    assert npair[0] >= 1 and tuple(pairs[:2]) == (1, 2)


def test_mklref_mssa(oracle, mklref):
    """mssa_opt_decompose / reconstruct_all / series_contributions (MKL/ssa_opt.h:3908-4283) with
    a registered test matrix."""
    rng = np.random.default_rng(11)
    Mch, N, L, k, p = 3, 400, 100, 8, 8
    X = oracle.config4_instance(rng, Mch=Mch, N=N)
    K = N - L + 1
    kp = min(k + p, Mch * L, K)
    Om = oracle.gaussian_omega(rng, K, kp)
    mklref.set_gaussian(mklref.omega_draws(Om))
    sig, U, V = np.zeros(k), np.zeros(Mch * L * k), np.zeros(K * k)
    grp = np.array([0, 1], dtype=np.int32)
    rec = np.zeros(Mch * N)
    con = np.zeros(Mch * k)
    n = mklref.lib.mkr_mssa(mklref.d(np.ascontiguousarray(X)), Mch, N, L, k, p, mklref.d(sig), mklref.d(U),
                            mklref.d(V), mklref.i(grp), 2, mklref.d(rec), mklref.d(con))
    assert n == k
    d = oracle.mssa_decompose(X, L, k, p, Om, q=0)
    _check_dec(sig, U.reshape(k, Mch * L).T, V.reshape(k, K).T, d)
    for m in range(Mch):
        ref = oracle.mssa_reconstruct(d, m, [0, 1], Mch, N, L)
        assert np.max(np.abs(rec[m * N:(m + 1) * N] - ref)) < 1e-9 * np.max(np.abs(ref))
    co = oracle.mssa_series_contributions(d, Mch, L)
    got = con.reshape(Mch, k) if con.size == Mch * k else con
    assert np.allclose(np.sort(got.ravel()), np.sort(co.ravel()), atol=1e-10)


@pytest.mark.parametrize("mode", ["plain", "weighted", "block_branch"])
def test_mklref_cadzow(oracle, mklref, mode):
    """ssa_opt_cadzow / _weighted (MKL/ssa_opt.h:3165-3315): every iteration re-initialises a
    context, whose fresh stream restarts the registered draws (the oracle takes one Omega)."""
    N = 400
    x = oracle.reference_test_signal(N)
    if mode == "block_branch":
        L, rank = 30, 8  # rank + 8 >= min(L, K) / 2: block power, 3 iterations
    else:
        L, rank = 100, 4
    K = N - L + 1
    out = np.zeros(N)
    its = np.zeros(1, dtype=np.int32)
    fd, cv = np.zeros(1), np.zeros(1)
    if mode == "block_branch":
        u = np.random.default_rng(2).random(K * rank)
        mklref.set_uniform(u)
        Om = (u - 0.5).reshape(rank, K).T
    else:
        kp = min(rank + 8, L, K)
        Om = oracle.gaussian_omega(np.random.default_rng(2), K, kp)
        mklref.set_gaussian(mklref.omega_draws(Om))
    alpha = 0.7 if mode == "weighted" else 1.0
    rc = mklref.lib.mkr_cadzow(mklref.d(x), N, L, rank, 6, 1e-12, 1 if mode == "weighted" else 0, alpha,
                               mklref.d(out), mklref.i(its), mklref.d(fd), mklref.d(cv))
    mklref.set_uniform(None)
    assert rc >= 1
    if mode == "weighted":
        y, it, diff, conv = oracle.cadzow_weighted(x, L, rank, 6, 1e-12, alpha, Om)
    else:
        y, it, diff, conv = oracle.cadzow(x, L, rank, 6, 1e-12, Om)
    assert its[0] == it
    # the block branch runs 3 unconverged block-power iterations per step, which amplify
    # rounding (see test_mklref_block_power): a 1e-6 relative bar there, FP64 rounding otherwise
    tol = 1e-6 if mode == "block_branch" else 1e-9
    assert abs(fd[0] - diff) < tol * max(diff, 1e-3)
    assert np.max(np.abs(out - y)) < tol * np.max(np.abs(y))


def test_mklref_cadzow_inplace(oracle, mklref):
    """ssa_opt_cadzow_inplace (MKL/ssa_opt.h:3319-3442): one context, so iteration i draws the
    next test matrix of the same stream."""
    N, L, rank, iters = 400, 100, 4, 5
    x = oracle.reference_test_signal(N)
    K = N - L + 1
    kp = min(rank + 8, L, K)
    rng = np.random.default_rng(9)
    oms = [oracle.gaussian_omega(rng, K, kp) for _ in range(iters)]
    mklref.set_gaussian(np.concatenate([mklref.omega_draws(o) for o in oms]))
    out = np.zeros(N)
    its = np.zeros(1, dtype=np.int32)
    fd, cv = np.zeros(1), np.zeros(1)
    rc = mklref.lib.mkr_cadzow(mklref.d(x), N, L, rank, iters, 1e-14, 2, 1.0, mklref.d(out), mklref.i(its),
                               mklref.d(fd), mklref.d(cv))
    assert rc == iters
    y_last, it, diff, conv, _ = oracle.cadzow_inplace(x, L, rank, iters, 1e-14, oms)
    assert its[0] == it
    assert abs(fd[0] - diff) < 1e-9 * max(diff, 1e-6)
    assert np.max(np.abs(out - y_last)) < 1e-9 * np.max(np.abs(y_last))


def test_mklref_gapfill(oracle, mklref):
    """ssa_opt_gapfill (MKL/ssa_opt.h:3498-3683): every iteration a fresh context, the same
    registered test matrix each time."""
    N, L, rank = 500, 100, 4
    x = oracle.reference_test_signal(N)
    xg = x.copy()
    xg[[50, 51, 52, 200, 333, 334]] = np.nan
    K = N - L + 1
    kp = min(rank + 8, L, K)
    Om = oracle.gaussian_omega(np.random.default_rng(4), K, kp)
    mklref.set_gaussian(mklref.omega_draws(Om))
    y = xg.copy()
    its, cv, ng = (np.zeros(1, dtype=np.int32) for _ in range(3))
    fd = np.zeros(1)
    assert mklref.lib.mkr_gapfill(mklref.d(y), N, L, rank, 20, 1e-8, 0, mklref.i(its), mklref.d(fd),
                                  mklref.i(cv), mklref.i(ng)) == 0
    yo, it, diff, conv, n_gaps = oracle.gapfill(xg, L, rank, 20, 1e-8, lambda K_, kp_: Om)
    assert ng[0] == n_gaps == 6 and its[0] == it
    assert np.max(np.abs(y - yo)) < 1e-8 * np.max(np.abs(yo))


def test_mklref_gapfill_simple(oracle, mklref):
    """ssa_opt_gapfill_simple (MKL/ssa_opt.h:3685-3878): forecast/backcast blend; each segment
    decomposes in a fresh context (registered draws restart)."""
    N, L, rank = 600, 60, 4
    x = oracle.reference_test_signal(N)
    xg = x.copy()
    xg[300:306] = np.nan
    draws = np.random.default_rng(8).standard_normal(10 ** 5)
    mklref.set_gaussian(draws)
    y = xg.copy()
    its, cv, ng = (np.zeros(1, dtype=np.int32) for _ in range(3))
    fd = np.zeros(1)
    assert mklref.lib.mkr_gapfill(mklref.d(y), N, L, rank, 0, 0.0, 1, mklref.i(its), mklref.d(fd),
                                  mklref.i(cv), mklref.i(ng)) == 0

    def omega_fn(K, kp):
        return draws[:K * kp].reshape(kp, K).T

    yo, n_gaps = oracle.gapfill_simple(xg, L, rank, omega_fn)
    assert ng[0] == n_gaps == 6
    assert np.max(np.abs(y - yo)) < 1e-8 * np.max(np.abs(yo))


def test_mklref_parestimate(oracle, mklref):
    """ssa_opt_parestimate (MKL/ssa_opt.h:4304-4558; LAPACK dgels + dgeev) against the oracle's
    least-squares + eigenvalue restatement on the same decomposition (as sets)."""
    N, L, k, p = 600, 150, 6, 8
    t = np.arange(N)
    x = 3 * np.sin(2 * np.pi * t / 50) + 1.5 * np.sin(2 * np.pi * t / 20) + 0.01 * np.cos(0.3 * t)
    K = N - L + 1
    kp = min(k + p, L, K)
    Om = oracle.gaussian_omega(np.random.default_rng(6), K, kp)
    mklref.set_gaussian(mklref.omega_draws(Om))
    per, fr, mo, ra = (np.zeros(4) for _ in range(4))
    grp = np.array([0, 1, 2, 3], dtype=np.int32)
    assert mklref.lib.mkr_parestimate(mklref.d(x), N, L, k, p, mklref.i(grp), 4, mklref.d(per), mklref.d(fr),
                                      mklref.d(mo), mklref.d(ra)) == 4
    d = oracle.decompose_randomized(x, L, k, p, Om, q=0)
    o = oracle.parestimate(d, [0, 1, 2, 3], L)
    assert np.allclose(np.sort(np.abs(fr)), np.sort(np.abs(o["frequencies"])), atol=1e-9)
    assert np.allclose(np.sort(mo), np.sort(o["moduli"]), atol=1e-9)
    assert np.allclose(np.sort(per[np.isfinite(per)]), np.sort(o["periods"][np.isfinite(o["periods"])]),
                       rtol=1e-8)
    assert sorted(np.round(per).astype(int).tolist()) == [20, 20, 50, 50]
