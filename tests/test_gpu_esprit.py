"""ESPRIT (ssa_opt_parestimate, MKL/ssa_opt.h:4304-4558) on the GPU: against the oracle on the
same decomposition (eigenvalues compared as a set, since the eigen-solvers order them
differently), and the reference's own known-answer tests (MKL/test/ssa_opt_test.c:1055-1100,
2062-2113).

Tolerance: eigenvalues of Z within 1e-4 (the GPU factors are FP32: their perturbation ~1e-6 of
U moves the shift-invariance solution by about that times its conditioning)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import ssa_gpu

    return ssa_gpu


def as_eig(par):
    lam = par.moduli * np.exp(2j * np.pi * par.frequencies)
    return np.sort_complex(lam)


def test_esprit_vs_oracle(gpu, oracle):
    x, _, Om = oracle.config1(seed=0)
    N, L, k, p = 1000, 250, 10, 10
    d = oracle.decompose_randomized(x, L, k, p, Om[:, :k + p], q=2)
    gs = gpu.SSA(x, L)
    gs.decompose(k, oversampling=p, power_iters=2, omega=Om[:, :k + p])
    for group in ([1, 2], [0, 1, 2], [0, 1, 2, 3, 4, 5]):
        par = gs.parestimate(group)
        ref = oracle.parestimate(d, group, L)
        assert par.n_components == len(group)
        got, want = as_eig(par), np.sort_complex(ref["eig"])
        assert np.max(np.abs(got - want)) <= 1e-4, (group, got, want)
        np.testing.assert_allclose(par.rates, np.log(np.maximum(par.moduli, 1e-300)), atol=1e-12)
    assert gs.parestimate().n_components == k  # all components
    with pytest.raises(RuntimeError):
        gs.parestimate([0, 50])


def test_esprit_reference_known_answers(gpu):
    i = np.arange(500, dtype=np.float64)
    x = 3.0 * np.sin(2 * np.pi * i / 50.0) + 2.0 * np.sin(2 * np.pi * i / 20.0)
    s = gpu.SSA(x, 125)
    s.decompose(6, method="sequential", max_iter=100)
    par = s.parestimate([0, 1, 2, 3])
    assert par.n_components == 4
    assert any(abs(p - 50.0) < 2.0 for p in par.periods)
    assert any(abs(p - 20.0) < 2.0 for p in par.periods)
    for p_, m in zip(par.periods, par.moduli):
        if 5 < p_ < 100:
            assert m > 0.9
    i = np.arange(600, dtype=np.float64)
    x = 4.0 * np.sin(2 * np.pi * i / 60.0) + 2.0 * np.sin(2 * np.pi * i / 30.0) + np.sin(2 * np.pi * i / 15.0)
    s = gpu.SSA(x, 150)
    s.decompose(8, method="sequential", max_iter=100)
    par = s.parestimate([0, 1, 2, 3, 4, 5])
    for true_p in (60.0, 30.0, 15.0):
        err = min(abs(p_ - true_p) / true_p for p_, m in zip(par.periods, par.moduli) if m > 0.9)
        assert err < 0.05, true_p
    assert set(par.get_periodic_components(min_modulus=0.9)) == set(range(6))
