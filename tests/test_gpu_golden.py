"""The CUDA path against the reference's own product path, MKL/ssa_opt.h.

Golden vectors (tests/golden/mklref_q0_*.npz, made by tests/golden/make_golden.py) hold the
reference build's outputs — randomized decomposition at q = 0 (its only mode), reconstructions of
[0] and [1, 2], W-correlation, 50-step R-forecast of [0, 1, 2] — for the single-series workload
and three uneven-batch series. The GPU runs the same decomposition with the same host test
matrix (ssa_opt_decompose_randomized_ex, q = 0) through the C ABI.

Tolerances (the device computes the FFT convolutions and block products in FP32):
  * sigma: relative <= 1e-5 for components 0..2 (those the groups use) and every component whose
    relative gap to its neighbours exceeds 1e-3; <= 1e-4 for the rest;
  * reconstructions [0], [1, 2]: relative L2 <= 1e-5 when the group is separated from the other
    computed components by a relative gap > 1e-2 (else FP32 rounding / gap, as in
    tests/test_gpu_parity.py);
  * W-correlation: <= 1e-4 absolute on the leading 5 x 5 block, diagonal 1 within 1e-6;
  * forecast: relative L2 <= 1e-4.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))

CASES = sorted(p.stem for p in GOLDEN.glob("mklref_q0_*.npz"))


@pytest.fixture(scope="module")
def gpu():
    import ssa_gpu

    return ssa_gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def group_gap(sigma, group):
    out = [j for j in range(len(sigma)) if j not in group]
    return min(abs(sigma[i] - sigma[j]) / sigma[i] for i in group for j in out) if out else np.inf


def rec_tol(sigma, group):
    g = group_gap(sigma, group)
    return 1e-5 if g > 1e-2 else max(1e-5, 40 * 2.0 ** -24 / max(g, 1e-12))


@pytest.mark.parametrize("case", CASES)
def test_q0_matches_reference_build(gpu, case):
    import make_golden

    z = np.load(GOLDEN / f"{case}.npz")
    x, L, k, p = z["x"], int(z["L"]), int(z["k"]), int(z["p"])
    N = len(x)
    K = N - L + 1
    kp = min(k + p, L, K)
    Om = make_golden.omega(K, kp, int(z["omega_seed"]))
    s = gpu.SSA(x, L)
    s.decompose(k, oversampling=p, power_iters=0, omega=Om)
    sig = s.singular_values
    ref = z["sigma"]
    rel = np.abs(sig - ref) / ref
    gap = np.full(k, np.inf)
    d = np.abs(np.diff(ref)) / ref[:-1]
    gap[:-1] = np.minimum(gap[:-1], d)
    gap[1:] = np.minimum(gap[1:], d)
    tight = gap > 1e-3
    tight[:3] = True
    print(f"\n{case}: N={N} L={L} k={k}: sigma rel max {rel.max():.2e}, components 0-2 {rel[:3].max():.2e}")
    assert np.all(rel[tight] <= 1e-5), rel[tight].max()
    assert np.all(rel <= 1e-4)
    for g, key in (([0], "rec0"), ([1, 2], "rec12")):
        e = rel_l2(s.reconstruct(g), z[key])
        print(f"  group {g}: rel L2 {e:.2e} (bar {rec_tol(ref, g):.1e})")
        assert e <= rec_tol(ref, g)
    W = s.wcorr_matrix()
    assert np.max(np.abs(np.diag(W) - 1.0)) < 1e-6
    assert np.max(np.abs(W[:5, :5] - z["W"][:5, :5])) < 1e-4
    fc = s.forecast([0, 1, 2], int(z["h"]))
    e = rel_l2(fc, z["forecast"])
    print(f"  forecast [0,1,2] x{int(z['h'])}: rel L2 {e:.2e}")
    assert e <= 1e-4


def test_wcorr_consumers_vs_oracle(gpu, oracle):
    """ssa_opt_wcorr_pair, ssa_opt_component_stats and ssa_opt_find_periodic_pairs
    (MKL/ssa_opt.h:2551-2756) on the device decomposition, against their definitions evaluated by
    the oracle (pinned to the reference build in tests/test_oracle_mklref.py) on the oracle's
    decomposition with the same test matrix."""
    N, L, k, p = 1000, 250, 16, 10
    x, _, Om = oracle.config1(seed=1, N=N, L=L, k=k, p=p)
    d = oracle.decompose_randomized(x, L, k, p, Om, q=0)
    s = gpu.SSA(x, L)
    s.decompose(k, oversampling=p, power_iters=0, omega=Om)
    Wo = oracle.wcorr_matrix(d, N, L)
    for i, j in ((0, 0), (1, 2), (1, 3), (3, 4), (0, 5)):
        assert abs(s.wcorr(i, j) - Wo[i, j]) < 1e-4, (i, j, s.wcorr(i, j), Wo[i, j])
    st = s.component_stats()
    sg = d.sigma
    assert np.allclose(st["singular_values"], sg, rtol=1e-4)
    assert np.allclose(st["gaps"], sg[:-1] / sg[1:], rtol=2e-4)
    assert np.allclose(st["cumulative_var"], np.cumsum(sg ** 2) / np.sum(sg ** 2), atol=1e-5)
    ls = np.log(sg)
    assert st["second_diff"][0] == 0.0 and st["second_diff"][-1] == 0.0
    assert np.allclose(st["second_diff"][1:-1], ls[:-2] - 2 * ls[1:-1] + ls[2:], atol=1e-3)
    assert st["suggested_signal"] == int(np.argmax(sg[:-1] / sg[1:])) + 1
    pairs = s.find_periodic_pairs(max_pairs=8, sv_tol=0.1, wcorr_thresh=0.5)
    # greedy definition (MKL/ssa_opt.h:2697-2756) on the oracle's sigma and W
    used, want = set(), []
    for i in range(k - 1):
        if i in used or len(want) >= 8:
            continue
        for j in range(i + 1, k):
            if j in used:
                continue
            if abs(1 - sg[j] / sg[i]) > 0.1 or abs(Wo[i, j]) < 0.5:
                continue
            want.append((i, j))
            used |= {i, j}
            break
    assert pairs == want and (1, 2) in pairs


def test_reference_call_sequence_raw_ctypes(gpu, oracle):
    """The call sequence of the reference's Python wrapper (MKL/py/ssa_wrapper.py:630-851) with
    its argument types, against libssa.so directly: a 1024-byte context buffer, ssa_opt_init,
    ssa_opt_prepare(k, 8), ssa_opt_decompose_randomized(k, 8) with the library's own test
    matrix (the device generator's first draw, reproduced by the oracle), reconstruct, W and
    forecast, struct-free result reads through the getters."""
    import ctypes

    lib = ctypes.CDLL(str(Path(gpu.__file__).resolve().parent / "libssa.so"))
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    lib.ssa_opt_init.argtypes = [ctypes.c_void_p, dp, ctypes.c_int, ctypes.c_int]
    lib.ssa_opt_prepare.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.ssa_opt_decompose_randomized.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.ssa_opt_reconstruct.argtypes = [ctypes.c_void_p, ip, ctypes.c_int, dp]
    lib.ssa_opt_wcorr_matrix.argtypes = [ctypes.c_void_p, dp]
    lib.ssa_opt_forecast.argtypes = [ctypes.c_void_p, ip, ctypes.c_int, ctypes.c_int, dp]
    lib.ssa_opt_get_singular_values.argtypes = [ctypes.c_void_p, dp, ctypes.c_int]
    lib.ssa_opt_free.argtypes = [ctypes.c_void_p]
    N, L, k = 1000, 250, 20
    x, _, _ = oracle.config1(seed=4, N=N, L=L, k=k, p=8)
    buf = ctypes.create_string_buffer(1024)
    D = lambda a: a.ctypes.data_as(dp)  # noqa: E731
    I = lambda a: a.ctypes.data_as(ip)  # noqa: E731
    assert lib.ssa_opt_init(buf, D(x), N, L) == 0
    try:
        assert lib.ssa_opt_prepare(buf, k, 8) == 0
        assert lib.ssa_opt_decompose_randomized(buf, k, 8) == 0
        sig = np.zeros(k)
        assert lib.ssa_opt_get_singular_values(buf, D(sig), k) == k
        K = N - L + 1
        Om = oracle.device_gaussian(oracle.single_series_seed(0), K, k + 8)
        d = oracle.decompose_randomized(x, L, k, 8, Om, q=0)
        assert np.max(np.abs(sig[:3] - d.sigma[:3]) / d.sigma[:3]) < 1e-5
        rec = np.zeros(N)
        g = np.array([1, 2], dtype=np.int32)
        assert lib.ssa_opt_reconstruct(buf, I(g), 2, D(rec)) == 0
        assert rel_l2(rec, oracle.reconstruct(d, [1, 2], N, L)) <= 1e-5
        W = np.zeros(k * k)
        assert lib.ssa_opt_wcorr_matrix(buf, D(W)) == 0
        assert np.max(np.abs(W.reshape(k, k)[:3, :3] - oracle.wcorr_matrix(d, N, L)[:3, :3])) < 1e-4
        fc = np.zeros(30)
        g3 = np.array([0, 1, 2], dtype=np.int32)
        assert lib.ssa_opt_forecast(buf, I(g3), 3, 30, D(fc)) == 0
        assert rel_l2(fc, oracle.forecast(d, [0, 1, 2], 30, N, L)) <= 1e-4
    finally:
        lib.ssa_opt_free(buf)
