"""Shared fixtures: paths, the oracle module and the reference checker library.

GPU tests are marked ``gpu``; everything else runs on a CPU-only machine.
"""
import ctypes
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "singular-spectrum-analysis_b200"
ORACLE = ROOT / "oracle"
GOLDEN = Path(__file__).resolve().parent / "golden"

for p in (str(PKG), str(ORACLE)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import ssa_oracle

    return ssa_oracle


class RefLib:
    """ctypes view of oracle/_ref/libssa_ref.so (the reference's ssa_opt_ref.h behind
    oracle/ref_driver.c)."""

    def __init__(self, path: Path):
        self.lib = ctypes.CDLL(str(path))
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L = self.lib
        L.refdrv_default_state.restype = ctypes.c_uint64
        L.refdrv_omega.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, dp]
        L.refdrv_matvec.argtypes = [dp, ctypes.c_int, ctypes.c_int, dp, dp]
        L.refdrv_matvec_T.argtypes = [dp, ctypes.c_int, ctypes.c_int, dp, dp]
        L.refdrv_reconstruct.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp, ip,
                                         ctypes.c_int, dp]
        L.refdrv_wcorr.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp]
        L.refdrv_lrf.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp, ip,
                                 ctypes.c_int, dp, dp]
        L.refdrv_forecast.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp, ip,
                                      ctypes.c_int, ctypes.c_int, dp]
        L.refdrv_sequential.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        dp, dp, dp]
        L.refdrv_randomized.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_uint64, dp, dp, dp]
        L.refdrv_pipeline.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_uint64, ip, ip, ctypes.c_int, dp, dp, dp]

    @staticmethod
    def d(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    @staticmethod
    def i(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def build_checkers() -> bool:
    """Builds oracle/_ref/ with oracle/Makefile (which locates the reference sources: its
    SSA_REFERENCE_DIR, overridable from the environment). False when they are absent."""
    r = subprocess.run(["make", "-C", str(ORACLE)], capture_output=True, text=True)
    return r.returncode == 0


def reference_dir():
    """The reference tree's MKL/ directory as oracle/Makefile resolves it, or None."""
    r = subprocess.run(["make", "-s", "-C", str(ORACLE), "print-refdir"], capture_output=True, text=True)
    d = Path(r.stdout.strip()) if r.returncode == 0 and r.stdout.strip() else None
    return d if d is not None and d.is_dir() else None


@pytest.fixture(scope="session")
def reflib():
    so = ORACLE / "_ref" / "libssa_ref.so"
    if not so.exists() and not build_checkers():
        pytest.skip("reference checker library not built and reference sources absent")
    return RefLib(so)


class MklRef:
    """ctypes view of oracle/_ref/libssa_mklshim.so: the reference's own MKL/ssa_opt.h compiled
    against the MKL-compatibility shim (oracle/mklshim/), entry points of oracle/mklref_driver.c.
    Gaussian / uniform draws of the reference's VSL streams come from registered buffers."""

    def __init__(self, path: Path):
        self.lib = ctypes.CDLL(str(path))
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        c_int, c_double = ctypes.c_int, ctypes.c_double
        L = self.lib
        L.mklshim_set_gaussian.argtypes = [dp, ctypes.c_long]
        L.mklshim_set_uniform.argtypes = [dp, ctypes.c_long]
        L.mkr_randomized.argtypes = [dp, c_int, c_int, c_int, c_int, dp, dp, dp, dp]
        L.mkr_block.argtypes = [dp, c_int, c_int, c_int, c_int, c_int, dp, dp, dp]
        L.mkr_sequential.argtypes = [dp, c_int, c_int, c_int, c_int, dp, dp, dp]
        L.mkr_matvec.argtypes = [dp, c_int, c_int, dp, dp, c_int]
        L.mkr_pipeline.argtypes = [dp, c_int, c_int, c_int, c_int, ip, ip, c_int, dp, c_int, dp, ip, c_int,
                                   c_int, dp, dp, dp, dp]
        L.mkr_wcorr_consumers.argtypes = [dp, c_int, c_int, c_int, c_int, ip, ip, c_int, dp, dp, dp, dp, ip, ip,
                                          c_int, c_double, c_double, ip]
        L.mkr_mssa.argtypes = [dp, c_int, c_int, c_int, c_int, c_int, dp, dp, dp, ip, c_int, dp, dp]
        L.mkr_cadzow.argtypes = [dp, c_int, c_int, c_int, c_int, c_double, c_int, c_double, dp, ip, dp, dp]
        L.mkr_gapfill.argtypes = [dp, c_int, c_int, c_int, c_int, c_double, c_int, ip, dp, ip, ip]
        L.mkr_parestimate.argtypes = [dp, c_int, c_int, c_int, c_int, ip, c_int, dp, dp, dp, dp]
        L.mkr_dims.argtypes = [dp, c_int, c_int, ip, ip]
        self._gauss = self._unif = None

    @staticmethod
    def d(a):
        return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    @staticmethod
    def i(a):
        return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))

    def set_gaussian(self, draws):
        """Every VSL stream created afterwards reads these N(0,1) draws from their start."""
        self._gauss = None if draws is None else np.ascontiguousarray(draws, dtype=np.float64).ravel()
        self.lib.mklshim_set_gaussian(self.d(self._gauss), 0 if self._gauss is None else self._gauss.size)

    def set_uniform(self, draws):
        """Every VSL stream created afterwards reads these U[0, 1) draws from their start."""
        self._unif = None if draws is None else np.ascontiguousarray(draws, dtype=np.float64).ravel()
        self.lib.mklshim_set_uniform(self.d(self._unif), 0 if self._unif is None else self._unif.size)

    def exhausted(self) -> bool:
        return bool(self.lib.mklshim_draws_exhausted())

    @staticmethod
    def omega_draws(Om):
        """A K x kp test matrix in the order the reference draws it (column-major)."""
        return np.ascontiguousarray(np.asarray(Om, dtype=np.float64).T).ravel()

    def randomized(self, x, L, k, p, Om):
        x = np.ascontiguousarray(x, dtype=np.float64)
        N = len(x)
        K = N - L + 1
        self.set_gaussian(self.omega_draws(Om))
        sig, U, V, tv = np.zeros(k), np.zeros(L * k), np.zeros(K * k), ctypes.c_double()
        n = self.lib.mkr_randomized(self.d(x), N, L, k, p, self.d(sig), self.d(U), self.d(V), ctypes.byref(tv))
        assert n > 0 and not self.exhausted()
        return sig[:n], U[:L * n].reshape(n, L).T, V[:K * n].reshape(n, K).T, tv.value


@pytest.fixture(scope="session")
def mklref():
    so = ORACLE / "_ref" / "libssa_mklshim.so"
    if not so.exists() and not build_checkers():
        pytest.skip("shimmed reference library not built and reference sources absent")
    return MklRef(so)


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
