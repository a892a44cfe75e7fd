"""Request server (ssa_server_*): results against the FP64 oracle, the same alone and in a mix,
forecasts on resident series, ordering, rejection and eviction.

Tolerances as in the other parity tests: singular values relative <= 1e-5 where the relative gap
to the neighbours exceeds 1e-3 (1e-4 otherwise); reconstructions relative L2 <= 1e-5 for groups
separated by a relative gap > 1e-2, else max(1e-5, 40 * 2^-24 / gap); forecasts relative L2
<= 1e-4 (the recurrence amplifies the FP32 error of the LRF coefficients and the tail by up to
h (L-1) |R| terms). A request's generator seed is its own, so alone and in a mix it gets the same
test matrix and the results differ only in how FP64 Gram partials are chunked.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIG_TOL = 1e-5
REC_TOL = 1e-5
FC_TOL = 1e-4
P, Q = 10, 2


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


def oracle_dec(oracle, x, L, k, seed):
    N = len(x)
    K = N - L + 1
    kp = min(k + P, L, K)
    Om = oracle.device_gaussian(seed, K, kp)
    return oracle.decompose_randomized(x, L, k, P, Om, q=Q)


@pytest.mark.parametrize("pinned", [False, True, "mixed"])
def test_server_mixed_requests_vs_oracle(gpu, oracle, pinned):
    """Pageable buffers go through the staging areas, page-locked ones are read and written by the
    batch's gather and scatter kernels directly; "mixed" puts both kinds in one batch and within
    one request (a page-locked input with pageable outputs and the reverse, and requests whose
    outputs mix both, which are staged as a whole)."""
    rng = np.random.default_rng(21)
    shapes = [(800, 200, 12), (5000, 1250, 30), (12000, 3000, 20), (18000, 4500, 15), (2500, 625, 45),
              (70000, 17500, 14)]
    xs = [oracle.walk_sines(rng, N) for N, _, _ in shapes]
    srv = gpu.SSAServer(max_inflight=2, oversampling=P, power_iters=Q)
    R = gpu.Requests(3 * len(shapes), pinned=pinned)
    for i, ((N, L, k), x) in enumerate(zip(shapes, xs)):
        R.add_decompose(x, L, k, series_id=100 + i, seed=1000 + i)
    for i, ((N, L, k), x) in enumerate(zip(shapes, xs)):
        R.add_decompose(x, L, k, series_id=0, seed=2000 + i, wcorr=True)
    for i in range(len(shapes)):
        R.add_forecast(100 + i, 50)
    srv.run(R)
    assert np.all(R.statuses() == 0), R.statuses()
    for i, ((N, L, k), x) in enumerate(zip(shapes, xs)):
        d = oracle_dec(oracle, x, L, k, 1000 + i)
        r = R.result(i)
        check_sigma(r["sigma"], d.sigma)
        for gi, g in enumerate(([0], [1, 2])):
            assert rel_l2(r["groups"][gi], oracle.reconstruct(d, g, N, L)) <= rec_tol(d.sigma, g), (i, g)
        fc = R.result(2 * len(shapes) + i)["forecast"]
        fr = oracle.forecast(d, [0, 1, 2], 50, N, L)
        assert rel_l2(fc, fr) <= FC_TOL, (i, rel_l2(fc, fr))
        dw = oracle_dec(oracle, x, L, k, 2000 + i)
        rw = R.result(len(shapes) + i)
        check_sigma(rw["sigma"], dw.sigma)
        Wr = oracle.wcorr_matrix(dw, N, L)
        assert np.max(np.abs(np.diag(rw["W"]) - 1.0)) < 1e-6
        blk = [j for j in range(min(5, len(dw.sigma))) if group_gap(dw.sigma, [j]) > 1e-2]
        if blk:
            assert np.max(np.abs(rw["W"][np.ix_(blk, blk)] - Wr[np.ix_(blk, blk)])) < 1e-4
    st = srv.stats()
    assert st["completed"] == 3 * len(shapes) and st["forecasts"] == len(shapes)
    srv.close()


def test_server_alone_equals_in_mix(gpu, oracle):
    rng = np.random.default_rng(5)
    x = oracle.walk_sines(rng, 6000)
    L, k = 1500, 25
    srv = gpu.SSAServer(max_inflight=3, oversampling=P, power_iters=Q)
    A = gpu.Requests(2)
    A.add_decompose(x, L, k, series_id=7, seed=99)
    A.add_forecast(7, 40)
    srv.run(A)
    alone, fa = A.result(0), A.result(1)
    assert alone["status"] == 0 and fa["status"] == 0
    # the same two requests in the middle of a stream of 40 others of mixed size
    mix = oracle.config3_batch(40, seed=8, nmin=500, nmax=20000)
    M = gpu.Requests(42)
    for j, (xj, Lj, kj) in enumerate(mix[:20]):
        M.add_decompose(xj, Lj, kj, series_id=200 + j, seed=500 + j, wcorr=bool(j % 3 == 0))
    i0 = M.add_decompose(x, L, k, series_id=7, seed=99)
    i1 = M.add_forecast(7, 40)
    for j, (xj, Lj, kj) in enumerate(mix[20:]):
        M.add_decompose(xj, Lj, kj, series_id=300 + j, seed=600 + j)
    arrivals = np.cumsum(np.full(M.n, 2e-4))
    srv.run(M, arrivals)
    assert np.all(M.statuses() == 0)
    inmix, fm = M.result(i0), M.result(i1)
    check_sigma(inmix["sigma"], alone["sigma"])
    for gi, g in enumerate(([0], [1, 2])):
        assert rel_l2(inmix["groups"][gi], alone["groups"][gi]) <= rec_tol(alone["sigma"], g)
    assert rel_l2(fm["forecast"], fa["forecast"]) <= FC_TOL
    assert srv.stats()["batches"] >= 2
    srv.close()


def test_server_rejections_and_waiting(gpu, oracle):
    rng = np.random.default_rng(6)
    x = oracle.walk_sines(rng, 3000)
    srv = gpu.SSAServer(max_inflight=1)
    R = gpu.Requests(6)
    i_unknown = R.add_forecast(12345, 10)                  # never decomposed
    i_bad = R.add_decompose(np.zeros(140000), 100, 10, 1)   # N beyond the largest FFT length
    i_ok = R.add_decompose(x, 750, 20, series_id=2, seed=3)
    i_wait = R.add_forecast(2, 10)                          # arrives while its series is queued
    i_h = R.add_forecast(2, 0)                              # h out of range
    i_small = R.add_decompose(x, 750, 2, series_id=3, seed=4)  # k < 3: nothing to forecast from
    srv.run(R)
    st = R.statuses()
    assert st[i_unknown] == -1 and st[i_bad] == -1 and st[i_h] == -1
    assert st[i_ok] == 0 and st[i_wait] == 0 and st[i_small] == 0
    R2 = gpu.Requests(1)
    R2.add_forecast(3, 10)
    srv.run(R2)
    assert R2.statuses()[0] == -1
    srv.close()


def resident_bytes(N, L, k):
    """Device bytes of one resident series: R, tail, verticality, sigma and the signal (doubles,
    rounded to an even count), then U and V with leading dimensions rounded to 4 (floats)."""
    K = N - L + 1
    nd = 2 * (L - 1) + 1 + k + N
    nd += nd & 1
    r4 = lambda v: (v + 3) & ~3  # noqa: E731
    return 8 * nd + 4 * (r4(L) + r4(K)) * k


def test_server_evicts_beyond_resident_budget(gpu, oracle):
    rng = np.random.default_rng(7)
    N, L, k = 4000, 1000, 10
    # resident share = budget / 4
    budget = 4 << 20
    srv = gpu.SSAServer(hbm_budget_bytes=budget, max_inflight=2, oversampling=P, power_iters=Q)
    per = resident_bytes(N, L, k)
    n_fit = (budget // 4) // per
    n = n_fit + 15
    R = gpu.Requests(n, keep_outputs=False)
    for i in range(n):
        R.add_decompose(oracle.walk_sines(rng, N), L, k, series_id=i, seed=i)
    srv.run(R)
    assert np.all(R.statuses() == 0)
    st = srv.stats()
    assert st["resident_bytes"] == n_fit * per <= st["resident_budget"]
    assert st["evictions"] == n - n_fit
    F = gpu.Requests(2)
    F.add_forecast(0, 5)       # least recently used: evicted
    F.add_forecast(n - 1, 5)   # most recent: resident
    srv.run(F)
    assert list(F.statuses()) == [-1, 0]
    srv.close()


def cadzow_from_factors(oracle, x, d, L, rank, iters, tol):
    """Cadzow on x whose first projection is the reconstruction of components 0..rank-1 of the
    decomposition d; later iterations as ssa_opt_cadzow (a fresh context each: the first-call test
    matrix, q = 0, oversampling 8). Returns (signal, iterations, final_diff)."""
    N = len(x)
    K = N - L + 1
    xn = float(np.linalg.norm(x)) or 1.0
    y = oracle.reconstruct(d, list(range(rank)), N, L)
    diff = float(np.linalg.norm(y - x)) / xn
    it = 1
    Om = oracle.device_gaussian(oracle.single_series_seed(0), K, min(rank + 8, L, K))
    while it < iters and diff >= tol:
        dec = oracle.decompose_randomized(y, L, rank, 8, Om, q=0)
        yn = oracle.reconstruct(dec, list(range(rank)), N, L)
        diff = float(np.linalg.norm(yn - y)) / xn
        y = yn
        it += 1
    return y, it, diff


def _followups(gpu, R, shapes):
    """Follow-ups on the resident series 7 (reconstruct decomposition) and 8 (W decomposition)."""
    (N7, L7, k7), (N8, L8, k8) = shapes
    i = {}
    i["rec"] = R.add_reconstruct(7, N7, [0, 3, 4])
    i["rec_skip"] = R.add_reconstruct(8, N8, [1, 2, 99])  # out-of-range indices are skipped
    i["fc"] = R.add_forecast(8, 30, group=[0, 1, 2, 3])
    i["fc_default"] = R.add_forecast(7, 30)
    i["cz"] = R.add_cadzow(4, max_iter=5, tol=1e-14, series_id=7, N=N7)
    return i


def test_server_followups_vs_oracle_alone_and_in_mix(gpu, oracle):
    """RECONSTRUCT(group), FORECAST(group, h) and CADZOW on resident series: results against the
    oracle on the same decompositions, the same alone and inside a 40-request mix, and no
    decomposition issued for them (ssa_server_stats.decompositions unchanged)."""
    rng = np.random.default_rng(31)
    shapes = [(6000, 1500, 20), (9000, 2250, 16)]
    xs = [oracle.walk_sines(rng, N) for N, _, _ in shapes]
    srv = gpu.SSAServer(max_inflight=2, oversampling=P, power_iters=Q)
    D = gpu.Requests(2)
    D.add_decompose(xs[0], shapes[0][1], shapes[0][2], series_id=7, seed=77)
    D.add_decompose(xs[1], shapes[1][1], shapes[1][2], series_id=8, seed=88, wcorr=True)
    srv.run(D)
    assert np.all(D.statuses() == 0)
    st0 = srv.stats()
    A = gpu.Requests(5)
    ia = _followups(gpu, A, shapes)
    srv.run(A)
    st1 = srv.stats()
    assert np.all(A.statuses() == 0), A.statuses()
    assert st1["decompositions"] == st0["decompositions"] and st1["batches"] == st0["batches"]
    assert st1["followups"] - st0["followups"] == 4 and st1["cadzow_requests"] - st0["cadzow_requests"] == 1
    d7 = oracle_dec(oracle, xs[0], shapes[0][1], shapes[0][2], 77)
    d8 = oracle_dec(oracle, xs[1], shapes[1][1], shapes[1][2], 88)
    (N7, L7, _), (N8, L8, _) = shapes
    rec = A.result(ia["rec"])["out"]
    assert rel_l2(rec, oracle.reconstruct(d7, [0, 3, 4], N7, L7)) <= rec_tol(d7.sigma, [0, 3, 4])
    rec2 = A.result(ia["rec_skip"])["out"]
    assert rel_l2(rec2, oracle.reconstruct(d8, [1, 2], N8, L8)) <= rec_tol(d8.sigma, [1, 2])
    fc = A.result(ia["fc"])["forecast"]
    assert rel_l2(fc, oracle.forecast(d8, [0, 1, 2, 3], 30, N8, L8)) <= FC_TOL
    fc7 = A.result(ia["fc_default"])["forecast"]
    assert rel_l2(fc7, oracle.forecast(d7, [0, 1, 2], 30, N7, L7)) <= FC_TOL
    cz = A.result(ia["cz"])
    y_ref, it_ref, diff_ref = cadzow_from_factors(oracle, xs[0], d7, L7, 4, 5, 1e-14)
    assert cz["iterations"] == it_ref
    assert rel_l2(cz["out"], y_ref) <= 1e-4
    assert abs(cz["final_diff"] - diff_ref) <= 1e-5
    # the same follow-ups in the middle of a stream of 40 other requests of mixed size
    mix = oracle.config3_batch(40, seed=9, nmin=500, nmax=20000)
    M = gpu.Requests(45)
    for j, (xj, Lj, kj) in enumerate(mix[:20]):
        M.add_decompose(xj, Lj, kj, series_id=400 + j, seed=700 + j, wcorr=bool(j % 3 == 0))
    im = _followups(gpu, M, shapes)
    for j, (xj, Lj, kj) in enumerate(mix[20:]):
        M.add_decompose(xj, Lj, kj, series_id=500 + j, seed=800 + j)
    srv.run(M, np.cumsum(np.full(M.n, 2e-4)))
    assert np.all(M.statuses() == 0), M.statuses()
    for key in ("rec", "rec_skip"):
        assert rel_l2(M.result(im[key])["out"], A.result(ia[key])["out"]) <= 1e-6
    for key in ("fc", "fc_default"):
        assert rel_l2(M.result(im[key])["forecast"], A.result(ia[key])["forecast"]) <= 1e-6
    assert rel_l2(M.result(im["cz"])["out"], cz["out"]) <= 1e-6
    srv.close()


def test_server_cadzow_new_series_and_followup_rejections(gpu, oracle):
    """CADZOW on a new series (its own signal) equals ssa_opt_cadzow; follow-ups fail on series
    that are not resident, empty groups, forecast groups with no component, and ranks above k'."""
    rng = np.random.default_rng(32)
    x = oracle.walk_sines(rng, 3000)
    L = 750
    srv = gpu.SSAServer(max_inflight=1, oversampling=P, power_iters=Q)
    R = gpu.Requests(8)
    i_new = R.add_cadzow(5, max_iter=4, tol=1e-14, x=x, L=L)
    i_dec = R.add_decompose(x, L, 6, series_id=11, seed=5)
    i_unknown = R.add_reconstruct(4242, 3000, [0])
    i_empty = R.add_reconstruct(11, 3000, [])
    i_nocomp = R.add_forecast(11, 10, group=[50, 60])
    i_rank = R.add_cadzow(7, max_iter=3, series_id=11, N=3000)  # k' = 6
    i_ok = R.add_reconstruct(11, 3000, [0, 1])
    srv.run(R)
    st = R.statuses()
    assert st[i_new] == 0 and st[i_dec] == 0 and st[i_ok] == 0
    assert st[i_unknown] == -1 and st[i_empty] == -1 and st[i_nocomp] == -1 and st[i_rank] == -1
    ref = gpu.cadzow(x, L, 5, max_iter=4, tol=1e-14)
    r = R.result(i_new)
    assert r["iterations"] == ref.iterations
    assert rel_l2(r["out"], ref.signal) <= 1e-6
    srv.close()


def test_server_short_bucket_completes_ahead_of_batch(gpu, oracle):
    """One batch of short series (N = 1000, real FFT length 1024) and longer ones (N = 30000,
    length 32768), offered together: the batch is ordered by FFT-length bucket and each bucket's
    requests complete when that bucket is done, so every short one finishes before any long one
    of the same batch; results against the oracle for one of each."""
    rng = np.random.default_rng(21)
    short = [oracle.walk_sines(rng, 1000) for _ in range(160)]
    long_ = [oracle.walk_sines(rng, 30000) for _ in range(24)]
    srv = gpu.SSAServer(max_inflight=1, oversampling=P, power_iters=Q)
    R = gpu.Requests(len(short) + len(long_) + 1)
    # a long-class series first holds the only batch slot, so that the others, submitted
    # meanwhile, form one batch
    R.add_decompose(oracle.walk_sines(rng, 90000), 22500, 40, series_id=4999, seed=1)
    idx_s, idx_l = [], []
    for j in range(max(len(short), len(long_))):  # interleaved arrival order
        if j < len(long_):
            idx_l.append(R.add_decompose(long_[j], 7500, 30, series_id=5000 + j, seed=900 + j))
        if j < len(short):
            idx_s.append(R.add_decompose(short[j], 250, 20, series_id=6000 + j, seed=700 + j))
    srv.run(R, np.zeros(R.n))
    assert np.all(R.statuses() == 0)
    assert srv.stats()["batches"] == 2
    _, td = R.times()
    assert td[idx_s].max() < td[idx_l].min(), (td[idx_s].max(), td[idx_l].min())
    for i, x, L, k, sd in ((idx_s[3], short[3], 250, 20, 703), (idx_l[2], long_[2], 7500, 30, 902)):
        d = oracle_dec(oracle, x, L, k, sd)
        res = R.result(i)
        check_sigma(res["sigma"], d.sigma)
        for gi, g in enumerate(([0], [1, 2])):
            assert rel_l2(res["groups"][gi], oracle.reconstruct(d, g, len(x), L)) <= rec_tol(d.sigma, g)
    srv.close()
