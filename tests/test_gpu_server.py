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


def test_server_evicts_beyond_resident_budget(gpu, oracle):
    rng = np.random.default_rng(7)
    N, L, k = 4000, 1000, 10
    # resident share = budget / 4; each resident series holds 2 (L - 1) + 1 doubles
    budget = 4 << 20
    srv = gpu.SSAServer(hbm_budget_bytes=budget, max_inflight=2, oversampling=P, power_iters=Q)
    per = 8 * (2 * (L - 1) + 1)
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
