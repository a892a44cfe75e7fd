"""W-correlation Gram on the tensor cores (tcgen05, split TF32, FP32 accumulation in TMEM)
against the FP64 CUDA-core path and the FP64 oracle, in the single-series API, the uniform batch
and the uneven batch.

Tolerances: tensor-core vs FP64 path, max |W_tc - W_fp64| <= 5e-6 (the split keeps ~21 bits
per product; partial sums run in FP32 over chunks of 1024+ time steps, ~sqrt(1024) 2^-24 = 2e-6
relative, measured 2.1e-6 at most); against the
oracle, the same bounds as the other parity tests (diagonal 1 within 1e-6, 1e-4 on the leading
well-separated block); the kernels' self-check record stays clean.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import ssa_gpu

    yield ssa_gpu
    ssa_gpu.set_wcorr_tensor_cores(True)


def group_gap(sigma, i):
    others = [abs(sigma[i] - sigma[j]) / sigma[i] for j in range(len(sigma)) if j != i]
    return min(others) if others else np.inf


def w_single(gpu, x, L, k, Om, tc):
    gpu.set_wcorr_tensor_cores(tc)
    s = gpu.SSA(x, L)
    s.decompose(k, oversampling=10, power_iters=2, omega=Om)
    return s.wcorr_matrix()


@pytest.mark.parametrize("N,L,k", [(1000, 250, 50), (5000, 1250, 20), (20000, 5000, 64 - 10), (70000, 17500, 12)])
def test_tc_wcorr_matches_fp64_and_oracle(gpu, oracle, N, L, k):
    rng = np.random.default_rng(N)
    x = oracle.walk_sines(rng, N)
    K = N - L + 1
    Om = rng.standard_normal((K, min(k + 10, L, K)))
    gpu.device_checks(reset=True)
    Wt = w_single(gpu, x, L, k, Om, True)
    Wf = w_single(gpu, x, L, k, Om, False)
    assert gpu.device_checks(reset=True)[0] == 0
    assert np.max(np.abs(Wt - Wf)) <= 5e-6, np.max(np.abs(Wt - Wf))
    d = oracle.decompose_randomized(x, L, k, 10, Om, q=2)
    Wr = oracle.wcorr_matrix(d, N, L)
    assert np.max(np.abs(np.diag(Wt) - 1.0)) < 1e-6
    blk = [i for i in range(min(6, k)) if group_gap(d.sigma, i) > 1e-2]
    if blk:
        assert np.max(np.abs(Wt[np.ix_(blk, blk)] - Wr[np.ix_(blk, blk)])) < 1e-4


def test_tc_wcorr_in_batches(gpu, oracle):
    B, N, L, k = 8, 4000, 1000, 30
    X = oracle.config2_batch(B, seed=11, N=N)
    out = {}
    for tc in (True, False):
        gpu.set_wcorr_tensor_cores(tc)
        ub = gpu.SSABatch(B, N, L, k, oversampling=10, power_iters=2)
        s_u, W_u, G_u = ub.run(X, seed=5)
        rb = gpu.SSARaggedBatch(oversampling=10, power_iters=2)
        mix = oracle.config3_batch(6, seed=13, nmin=500, nmax=90000)
        s_r, W_r, G_r = rb.run([m[0] for m in mix], [m[1] for m in mix], [m[2] for m in mix], seed=3)
        out[tc] = (s_u, W_u, G_u, s_r, W_r, G_r)
    a, b = out[True], out[False]
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])  # only W depends on the mode
    assert np.max(np.abs(a[1] - b[1])) <= 5e-6
    for s in range(len(a[4])):
        assert np.array_equal(a[3][s], b[3][s])
        assert np.max(np.abs(a[4][s] - b[4][s])) <= 5e-6, s
    assert gpu.device_checks(reset=True)[0] == 0


@pytest.mark.parametrize("N,L,k", [(1000, 250, 50), (20000, 5000, 54)])
def test_wcorr_gram_arithmetics_against_fp64(gpu, oracle, N, L, k):
    """The four W-correlation Gram arithmetics on the same decomposition: split TF32 and FP32
    within 5e-6 of the FP64 path (~21-22 bits per product, FP32 partial sums over chunks of
    1024+ steps), split BF16 within 1e-4 (hi, lo of 8 significant bits each: ~16 bits per
    product); every mode leaves sigma untouched and the diagonal at 1."""
    rng = np.random.default_rng(N + 1)
    x = oracle.walk_sines(rng, N)
    K = N - L + 1
    Om = rng.standard_normal((K, min(k + 10, L, K)))
    Ws, sig = {}, {}
    try:
        for mode in (gpu.WGRAM_FP64, gpu.WGRAM_TF32X3, gpu.WGRAM_BF16X3, gpu.WGRAM_FP32):
            gpu.set_wcorr_gram(mode)
            assert gpu.wcorr_gram() == mode
            s = gpu.SSA(x, L)
            s.decompose(k, oversampling=10, power_iters=2, omega=Om)
            Ws[mode], sig[mode] = s.wcorr_matrix(), s.singular_values.copy()
    finally:
        gpu.set_wcorr_gram(gpu.WGRAM_TF32X3)
    assert gpu.device_checks(reset=True)[0] == 0
    ref = Ws[gpu.WGRAM_FP64]
    err = {m: float(np.max(np.abs(W - ref))) for m, W in Ws.items()}
    print(f"\nN={N} k={k}: max |W - W_fp64|: " + ", ".join(f"{gpu.WGRAM_NAMES[m]} {e:.2e}" for m, e in err.items()))
    for m in Ws:
        assert np.array_equal(sig[m], sig[gpu.WGRAM_FP64])
        assert np.max(np.abs(np.diag(Ws[m]) - 1.0)) < 1e-6
    assert err[gpu.WGRAM_TF32X3] <= 5e-6 and err[gpu.WGRAM_FP32] <= 5e-6
    assert err[gpu.WGRAM_BF16X3] <= 1e-4
    with pytest.raises(ValueError):
        gpu.set_wcorr_gram(7)


def test_wcorr_gram_arithmetics_in_uneven_batch(gpu, oracle):
    """The same comparison through the uneven batch, series across single-CTA and cluster
    lengths."""
    mix = oracle.config3_batch(6, seed=17, nmin=500, nmax=70000)
    out = {}
    try:
        for mode in (gpu.WGRAM_FP64, gpu.WGRAM_TF32X3, gpu.WGRAM_BF16X3, gpu.WGRAM_FP32):
            gpu.set_wcorr_gram(mode)
            rb = gpu.SSARaggedBatch(oversampling=10, power_iters=2)
            out[mode] = rb.run([m[0] for m in mix], [m[1] for m in mix], [m[2] for m in mix], seed=9)
    finally:
        gpu.set_wcorr_gram(gpu.WGRAM_TF32X3)
    ref = out[gpu.WGRAM_FP64]
    for mode, bar in ((gpu.WGRAM_TF32X3, 5e-6), (gpu.WGRAM_FP32, 5e-6), (gpu.WGRAM_BF16X3, 1e-4)):
        for s in range(len(mix)):
            assert np.array_equal(out[mode][0][s], ref[0][s])
            assert np.max(np.abs(out[mode][1][s] - ref[1][s])) <= bar, (mode, s)
    assert gpu.device_checks(reset=True)[0] == 0


def test_rowmul_tensor_cores_match_cuda_cores(gpu, oracle):
    """Row products on the tensor cores (three-part TF32 split, six products, FP32 accumulation in
    TMEM) against the FP32 CUDA-core form, in the single-series API and the uneven batch: both
    round like an FP32 product, so sigma and the group reconstructions agree to ~1e-6 relative,
    and each stays within 1e-5 of the FP64 oracle (same device test matrices, q = 2)."""
    x, _, Om = oracle.config1(seed=3)
    N, L, k = 1000, 250, 50
    mix = oracle.config3_batch(8, seed=19, nmin=500, nmax=100000)
    res = {}
    try:
        for on in (False, True):
            gpu.set_rowmul_tensor_cores(on)
            assert gpu.rowmul_tensor_cores() == on
            s = gpu.SSA(x, L)
            s.decompose(k, oversampling=10, power_iters=2, omega=Om)
            rb = gpu.SSARaggedBatch(oversampling=10, power_iters=2, groups=[[0], [1, 2]])
            sig, W, G = rb.run([m[0] for m in mix], [m[1] for m in mix], [m[2] for m in mix], seed=5)
            res[on] = (s.singular_values.copy(), s.reconstruct([0]), s.reconstruct([1, 2]), sig, G)
    finally:
        gpu.set_rowmul_tensor_cores(False)
    assert gpu.device_checks(reset=True)[0] == 0
    a, b = res[True], res[False]
    d = oracle.decompose_randomized(x, L, k, 10, Om, q=2)
    rel = lambda u, v: float(np.linalg.norm(u - v) / np.linalg.norm(v))  # noqa: E731
    assert np.max(np.abs(a[0][:3] - b[0][:3]) / b[0][:3]) < 2e-6
    assert rel(a[1], b[1]) < 5e-6 and rel(a[2], b[2]) < 5e-6
    assert np.max(np.abs(a[0][:3] - d.sigma[:3]) / d.sigma[:3]) < 1e-5
    assert rel(a[1], oracle.reconstruct(d, [0], N, L)) < 1e-5
    assert rel(a[2], oracle.reconstruct(d, [1, 2], N, L)) < 1e-5
    worst = 0.0
    for i, (xs, Ls, ks) in enumerate(mix):
        kk = min(ks, len(a[3][i]))
        e = np.max(np.abs(a[3][i][:3] - b[3][i][:3]) / b[3][i][:3])
        worst = max(worst, e)
        assert e < 2e-6, (i, e)
        for g in range(2):
            assert rel(a[4][i][g], b[4][i][g]) < 5e-6, (i, g)
    print(f"\nrow products tensor vs CUDA cores: sigma 0-2 max rel {worst:.2e}")
