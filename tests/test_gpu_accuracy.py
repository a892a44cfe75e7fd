"""The 1e-5 bar without exemptions: on the single-series, uniform and uneven workloads, the
singular values of the components the groups use (0, 1, 2) and the reconstructions of groups [0]
and [1, 2] are within 1e-5 (relative, relative L2) of the FP64 restatement of the same algorithm
with the same device test matrix (q = 2), for every series checked, whatever the gaps between
singular values. (The parity tests elsewhere also check the trailing components, with a
gap-dependent bar: FP32 rounding over a relative gap g moves a component's vectors by ~u/g.)"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BAR = 1e-5
P, Q = 10, 2


@pytest.fixture(scope="module")
def gpu():
    import ssa_gpu

    return ssa_gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _check(oracle, x, L, k, seed_s, sig, groups):
    N = len(x)
    K = N - L + 1
    kk, kp = oracle.clamp_kp(L, K, k, P)
    d = oracle.decompose_randomized(x, L, kk, P, oracle.device_gaussian(seed_s, K, kp), q=Q)
    lead = min(3, kk)
    e_sig = float(np.max(np.abs(sig[:lead] - d.sigma[:lead]) / d.sigma[:lead]))
    e_rec = max(rel_l2(groups[gi], oracle.reconstruct(d, g, N, L)) for gi, g in enumerate(([0], [1, 2]))
                if max(g) < kk)
    return e_sig, e_rec


def test_uneven_batch_64_series_bar(gpu, oracle):
    """64 series of the uneven-batch workload (N log-uniform in [500, 20000], L = N/4, k in
    10..50, random-walk trend + 1-3 sinusoids + noise at SNR 0-15 dB)."""
    series = oracle.config3_batch(64, seed=12, nmin=500, nmax=20000)
    rb = gpu.SSARaggedBatch(oversampling=P, power_iters=Q, groups=[[0], [1, 2]])
    seed = 3
    sig, W, G = rb.run([x for x, _, _ in series], [L for _, L, _ in series], [k for _, _, k in series], seed=seed,
                       want_w=np.zeros(64, dtype=bool))
    worst = (0.0, 0.0)
    for s, (x, L, k) in enumerate(series):
        e = _check(oracle, x, L, k, oracle.series_seed(seed, s), sig[s], G[s])
        worst = (max(worst[0], e[0]), max(worst[1], e[1]))
        assert e[0] <= BAR and e[1] <= BAR, (s, len(x), L, k, e)
    print(f"\nuneven batch: sigma 0-2 max rel {worst[0]:.2e}, groups max rel L2 {worst[1]:.2e}")


def test_uniform_batch_bar(gpu, oracle):
    """Sixteen series of the uniform workload (N = 10000, L = 2500, k = 50)."""
    B, N, L, k = 16, 10000, 2500, 50
    X = oracle.config2_batch(B, seed=1, N=N)
    b = gpu.SSABatch(B, N, L, k, oversampling=P, power_iters=Q, groups=[[0], [1, 2]])
    seed = 4
    sig, W, G = b.run(X, seed=seed)
    for s in range(B):
        e = _check(oracle, X[s], L, k, oracle.series_seed(seed, s), sig[s], G[s])
        assert e[0] <= BAR and e[1] <= BAR, (s, e)


def test_single_series_bar(gpu, oracle):
    """The single-series workload (N = 1000, L = 250, k = 50) with its host test matrix."""
    x, _, Om = oracle.config1(seed=0)
    N, L, k = 1000, 250, 50
    d = oracle.decompose_randomized(x, L, k, P, Om, q=Q)
    s = gpu.SSA(x, L)
    s.decompose(k, oversampling=P, power_iters=Q, omega=Om)
    sig = s.singular_values
    assert np.max(np.abs(sig[:3] - d.sigma[:3]) / d.sigma[:3]) <= BAR
    for g in ([0], [1, 2]):
        assert rel_l2(s.reconstruct(g), oracle.reconstruct(d, g, N, L)) <= BAR
