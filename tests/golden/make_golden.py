"""Generates the golden vectors in this directory from the reference's own product path.

The reference's MKL/ssa_opt.h, compiled unmodified against the MKL-compatibility shim
(oracle/Makefile -> oracle/_ref/libssa_mklshim.so), runs its randomized decomposition
(q = 0, the reference's only mode, ssa_opt.h:1685-1763) with a registered Gaussian test matrix,
then reconstruct [0] and [1, 2] (:2325-2400), W-correlation (:2407-2548) and the R-forecast of
group [0, 1, 2] (:2843-2867). Each case stores its signal, shape, the seed of its test matrix and
the outputs. Run from the repository root: ``python tests/golden/make_golden.py``.

Cases: the single-series workload (N = 1000, L = 250, k = 50, p = 10; its own generator's
test matrix) and three series of the uneven-batch generator (seed 2; N 1598, 2686, 5831) whose test
matrices come from ``omega(K, kp, omega_seed)`` below (not stored: regenerated by the tests).
The GPU parity tests (tests/test_gpu_golden.py) run the CUDA path with the same test matrices and
compare.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))

import ssa_oracle as O  # noqa: E402
from conftest import MklRef, build_checkers  # noqa: E402

H_FORECAST = 50


def omega(K: int, kp: int, omega_seed: int) -> np.ndarray:
    """The K x kp Gaussian test matrix of a case (-1: the single-series workload's own)."""
    if omega_seed < 0:
        return O.config1(seed=0, N=1000, L=250, k=50, p=10)[2][:, :kp]
    return O.gaussian_omega(np.random.default_rng(omega_seed), K, kp)


def cases():
    x, _, _ = O.config1(seed=0, N=1000, L=250, k=50, p=10)
    yield "config1", x, 250, 50, 10, -1
    rng = np.random.default_rng(2)
    for i in range(3):
        N = int(round(np.exp(rng.uniform(np.log(1000), np.log(6000)))))
        L = max(2, int(round(N / 4)))
        k = int(rng.integers(10, 51))
        x = O.walk_sines(rng, N)
        yield f"uneven{i}", x, L, k, 10, 100 + i


def main():
    so = ROOT / "oracle" / "_ref" / "libssa_mklshim.so"
    if not so.exists() and not build_checkers():
        raise SystemExit("shimmed reference library not available")
    ref = MklRef(so)
    for name, x, L, k, p, oseed in cases():
        N = len(x)
        K = N - L + 1
        Om = omega(K, O.clamp_kp(L, K, k, p)[1], oseed)
        ref.set_gaussian(ref.omega_draws(Om))
        groups = np.array([0, 1, 2], dtype=np.int32)
        sizes = np.array([1, 2], dtype=np.int32)
        rec = np.zeros(2 * N)
        W = np.zeros(k * k)
        fc = np.zeros(H_FORECAST)
        sig = np.zeros(k)
        fg = np.array([0, 1, 2], dtype=np.int32)
        n = ref.lib.mkr_pipeline(ref.d(x), N, L, k, p, ref.i(groups), ref.i(sizes), 2, ref.d(rec), 1, ref.d(W),
                                 ref.i(fg), 3, H_FORECAST, ref.d(fc), None, None, ref.d(sig))
        assert n == k and not ref.exhausted(), name
        np.savez_compressed(HERE / f"mklref_q0_{name}.npz", x=x, L=L, k=k, p=p, omega_seed=oseed,
                            sigma=sig, rec0=rec[:N], rec12=rec[N:], W=W.reshape(k, k), forecast=fc,
                            h=H_FORECAST)
        print(name, N, L, k, f"sigma0 {sig[0]:.6g}")


if __name__ == "__main__":
    main()
