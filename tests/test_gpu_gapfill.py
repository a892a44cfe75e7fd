"""Gap filling (ssa_opt_gapfill / ssa_opt_gapfill_simple, MKL/ssa_opt.h:3440-3878) on the GPU
against the oracle with the same test matrices (a fresh context's first generated matrix), and
the reference's own acceptance bars (MKL/test/ssa_opt_test.c:902-1000).

Tolerances: filled values within 1e-4 of the oracle's relative to the signal's peak (FP32
reconstruction and forecast noise is ~1e-6; the iterative comparison stops at a change of
1e-5 so that both converge on the same iteration or a neighbouring one). The reference's
1e-8 stopping rule is below FP32 resolution, so there the bars are the reference test's
(all gaps filled, RMSE < 0.5, n_gaps reported, at least one iteration)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import ssa_gpu

    return ssa_gpu


def signal(N, two_tones=True):
    i = np.arange(N, dtype=np.float64)
    s = np.sin(2 * np.pi * i / 50.0) + 0.02 * i
    if two_tones:
        s += 0.5 * np.sin(2 * np.pi * i / 20.0)
    return s


def omega(oracle):
    return lambda K, kp: oracle.device_gaussian(oracle.single_series_seed(0), K, kp)


def test_gapfill_iterative_vs_oracle(gpu, oracle):
    N, L, rank = 500, 100, 6
    true = signal(N)
    x = true.copy()
    x[50:65] = np.nan
    x[150:170] = np.nan
    r = gpu.gapfill(x, L, rank, max_iter=30, tol=1e-5)
    y, it, diff, conv, ng = oracle.gapfill(x, L, rank, 30, 1e-5, omega(oracle))
    assert r.n_gaps == ng == 35 and r.converged and conv
    assert abs(r.iterations - it) <= 1
    gaps = np.isnan(x)
    assert np.array_equal(r.signal[~gaps], x[~gaps])
    assert np.max(np.abs(r.signal[gaps] - y[gaps])) <= 1e-4 * np.abs(true).max()
    # the reference's bars at its own stopping rule
    r8 = gpu.gapfill(x, L, rank, max_iter=30, tol=1e-8)
    assert r8.n_gaps == 35 and r8.iterations > 0 and not np.isnan(r8.signal).any()
    assert np.sqrt(np.mean((r8.signal[gaps] - true[gaps]) ** 2)) < 0.5


def test_gapfill_simple_vs_oracle(gpu, oracle):
    N, L, rank = 500, 100, 6
    true = signal(N, two_tones=False)
    x = true.copy()
    x[200:220] = np.nan
    r = gpu.gapfill(x, L, rank, method="simple")
    y, ng = oracle.gapfill_simple(x, L, rank, omega(oracle))
    assert r.n_gaps == ng == 20 and r.iterations == 1 and r.converged
    assert not np.isnan(r.signal).any()
    assert np.max(np.abs(r.signal - y)) <= 1e-4 * np.abs(true).max()
    # runs too close to an end for one side: the other side's forecast alone (a left run's right
    # segment that still holds the later run gives none either); a run with neither side long
    # enough takes the mean of its neighbours
    for runs in (((30, 40),), ((470, 480),), ((30, 40), (470, 480))):
        x2 = true.copy()
        for lo, hi in runs:
            x2[lo:hi] = np.nan
        r2 = gpu.gapfill(x2, L, rank, method="simple")
        y2, _ = oracle.gapfill_simple(x2, L, rank, omega(oracle))
        assert not np.isnan(r2.signal).any()
        assert np.max(np.abs(r2.signal - y2)) <= 1e-4 * np.abs(true).max(), runs
    x3 = signal(120, two_tones=False)
    x3[55:60] = np.nan
    r3 = gpu.gapfill(x3, 100, 6, method="simple")
    np.testing.assert_allclose(r3.signal[55:60], 0.5 * (x3[54] + x3[60]))


def test_gapfill_edges(gpu, oracle):
    x = signal(300)
    r = gpu.gapfill(x, 60, 4)
    assert r.n_gaps == 0 and r.iterations == 0 and r.converged
    np.testing.assert_array_equal(r.signal, x)
    y = x.copy()
    y[:250] = np.nan  # fewer valid points than L + rank
    with pytest.raises(RuntimeError):
        gpu.gapfill(y, 60, 4)
    with pytest.raises(RuntimeError):
        gpu.gapfill(x, 300, 4)  # L > N - 1
    with pytest.raises(ValueError):
        gpu.gapfill(x, 60, 4, method="nope")
