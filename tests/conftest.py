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


@pytest.fixture(scope="session")
def reflib():
    so = ORACLE / "_ref" / "libssa_ref.so"
    if not so.exists():
        ref = Path("/root/reference/MKL/ssa_opt_ref.h")
        if not ref.exists():
            pytest.skip("reference checker library not built and reference sources absent")
        subprocess.run(["make", "-C", str(ORACLE)], check=True, capture_output=True)
    return RefLib(so)


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
