"""Python interface of the B200 SSA library (libssa.so in this directory).

Mirrors the classes and functions of SSA-Opt's ctypes wrapper (MKL/py/ssa_wrapper.py: ``SSA``
:600-1202, ``MSSA`` :1208-1371, ``cadzow`` :415-489) with the same method names, argument
meaning and error behaviour (``ValueError`` on a failed init, ``RuntimeError`` on a failed
call), and adds what the reference wrapper cannot express: power iterations and a caller-supplied
Gaussian test matrix for the randomized decomposition, and the batched pipeline (``SSABatch``).

Every numerical call runs on the GPU through the C ABI of libssa.so; there is no CPU path.
Importing this module raises ``ImportError`` when libssa.so has not been built.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import List, Optional, Sequence, Tuple

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libssa.so"
if not LIB_PATH.exists():
    raise ImportError(f"{LIB_PATH} is missing: run build.py (nvcc, sm_100a) first")

# 32 hardware work queues for the bucket and batch streams (read at CUDA context creation; the
# library's load-time default does the same for C callers)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
_lib = ctypes.CDLL(str(LIB_PATH))

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int_p = ctypes.POINTER(ctypes.c_int)


class _Opaque1024(ctypes.Structure):
    _fields_ = [("_opaque", ctypes.c_char * 1024)]


class _SSA_LRF(ctypes.Structure):
    _fields_ = [("R", c_double_p), ("L", ctypes.c_int), ("verticality", ctypes.c_double), ("valid", ctypes.c_bool)]


class _ComponentStats(ctypes.Structure):
    """SSA_ComponentStats (MKL/ssa_opt.h:228-248)."""
    _fields_ = [("n", ctypes.c_int), ("singular_values", ctypes.POINTER(ctypes.c_double)),
                ("log_sv", ctypes.POINTER(ctypes.c_double)), ("gaps", ctypes.POINTER(ctypes.c_double)),
                ("cumulative_var", ctypes.POINTER(ctypes.c_double)),
                ("second_diff", ctypes.POINTER(ctypes.c_double)), ("suggested_signal", ctypes.c_int),
                ("gap_threshold", ctypes.c_double)]


class _SSA_CadzowResult(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("final_diff", ctypes.c_double), ("converged", ctypes.c_double)]


class _BatchResults(ctypes.Structure):
    _fields_ = [("sigma", ctypes.c_void_p), ("W", ctypes.c_void_p), ("groups", ctypes.c_void_p),
                ("recon", ctypes.c_void_p), ("ld_recon", ctypes.c_longlong), ("status", ctypes.c_void_p),
                ("stream", ctypes.c_void_p)]


_P = ctypes.POINTER(_Opaque1024)


def _sig(name, restype, *argtypes):
    f = getattr(_lib, name)
    f.restype = restype
    f.argtypes = list(argtypes)
    return f


_I, _D, _V = ctypes.c_int, ctypes.c_double, None
_sig("ssa_opt_init", _I, _P, c_double_p, _I, _I)
_sig("ssa_opt_free", _V, _P)
_sig("ssa_opt_prepare", _I, _P, _I, _I)
_sig("ssa_opt_free_prepared", _V, _P)
_sig("ssa_opt_update_signal", _I, _P, c_double_p)
_sig("ssa_opt_decompose", _I, _P, _I, _I)
_sig("ssa_opt_decompose_block", _I, _P, _I, _I, _I)
_sig("ssa_opt_decompose_randomized", _I, _P, _I, _I)
_sig("ssa_opt_decompose_randomized_ex", _I, _P, _I, _I, _I, c_double_p)
_sig("ssa_opt_decompose_block_ex", _I, _P, _I, _I, _I, c_double_p)
_sig("ssa_opt_reconstruct", _I, _P, c_int_p, _I, c_double_p)
_sig("ssa_opt_cache_ffts", _I, _P)
_sig("ssa_opt_forecast", _I, _P, c_int_p, _I, _I, c_double_p)
_sig("ssa_opt_forecast_full", _I, _P, c_int_p, _I, _I, c_double_p)
_sig("ssa_opt_vforecast", _I, _P, c_int_p, _I, _I, c_double_p)
_sig("ssa_opt_vforecast_full", _I, _P, c_int_p, _I, _I, c_double_p)
_sig("ssa_opt_vforecast_fast", _I, _P, c_int_p, _I, c_double_p, _I, _I, c_double_p)
_sig("ssa_opt_compute_lrf", _I, _P, c_int_p, _I, ctypes.POINTER(_SSA_LRF))
_sig("ssa_opt_lrf_free", _V, ctypes.POINTER(_SSA_LRF))
_sig("ssa_opt_forecast_with_lrf", _I, ctypes.POINTER(_SSA_LRF), c_double_p, _I, _I, c_double_p)
_sig("ssa_opt_wcorr_matrix", _I, _P, c_double_p)
_sig("ssa_opt_wcorr_pair", _D, _P, _I, _I)
_sig("ssa_opt_variance_explained", _D, _P, _I, _I)
_sig("ssa_opt_find_periodic_pairs", _I, _P, c_int_p, _I, _D, _D)
_sig("ssa_opt_component_stats", _I, _P, ctypes.POINTER(_ComponentStats))
_sig("ssa_opt_component_stats_free", _V, ctypes.POINTER(_ComponentStats))
_sig("ssa_opt_get_trend", _I, _P, c_double_p)
_sig("ssa_opt_get_noise", _I, _P, _I, c_double_p)
_sig("ssa_opt_get_singular_values", _I, _P, c_double_p, _I)
_sig("ssa_opt_get_eigenvalues", _I, _P, c_double_p, _I)
_sig("ssa_opt_get_total_variance", _D, _P)
_sig("ssa_opt_hankel_matvec_dev", _I, _P, c_double_p, c_double_p)
_sig("ssa_opt_hankel_matvec_T_dev", _I, _P, c_double_p, c_double_p)
_sig("ssa_opt_cadzow", _I, c_double_p, _I, _I, _I, _I, _D, c_double_p, ctypes.POINTER(_SSA_CadzowResult))
_sig("ssa_opt_cadzow_weighted", _I, c_double_p, _I, _I, _I, _I, _D, _D, c_double_p,
     ctypes.POINTER(_SSA_CadzowResult))
_sig("mssa_opt_init", _I, _P, c_double_p, _I, _I, _I)
_sig("mssa_opt_decompose", _I, _P, _I, _I)
_sig("mssa_opt_decompose_ex", _I, _P, _I, _I, _I, c_double_p)
_sig("mssa_opt_reconstruct", _I, _P, _I, c_int_p, _I, c_double_p)
_sig("mssa_opt_reconstruct_all", _I, _P, c_int_p, _I, c_double_p)
_sig("mssa_opt_series_contributions", _I, _P, c_double_p)
_sig("mssa_opt_variance_explained", _D, _P, _I, _I)
_sig("mssa_opt_free", _V, _P)
_sig("ssa_opt_copy_factors", _I, _P, c_double_p, c_double_p)
_sig("ssa_opt_extend", _I, _P, _I, _I)
_sig("mssa_opt_copy_factors", _I, _P, c_double_p, c_double_p, c_double_p)
_sig("ssa_opt_cadzow_inplace", _I, _P, _I, _I, _D, ctypes.POINTER(_SSA_CadzowResult))
_sig("ssa_b200_kernel_launches", ctypes.c_ulonglong)
_sig("ssa_b200_sizeof_ssa_opt", _I)
_sig("ssa_batch_create", _I, ctypes.POINTER(ctypes.c_void_p), _I, _I, _I, _I, _I, _I, c_int_p, c_int_p, _I)
_sig("ssa_batch_destroy", _V, ctypes.c_void_p)
_sig("ssa_batch_run", _I, ctypes.c_void_p, c_double_p, _I, ctypes.c_uint64, c_double_p, c_double_p, c_double_p)
_sig("ssa_batch_run_device", _I, ctypes.c_void_p, ctypes.c_void_p, _I, ctypes.c_uint64)
_sig("ssa_batch_sync", _I, ctypes.c_void_p)
_sig("ssa_batch_device_results", _I, ctypes.c_void_p, ctypes.POINTER(_BatchResults))
_sig("ssa_batch_set_profiling", _I, ctypes.c_void_p, _I)
_sig("ssa_batch_status", _I, ctypes.c_void_p, c_int_p, _I)
_sig("ssa_batch_profile", _I, ctypes.c_void_p, c_double_p, ctypes.POINTER(ctypes.c_longlong), _I)

_sig("ssa_b200_set_wcorr_tensor_cores", _V, _I)
_sig("ssa_b200_wcorr_tensor_cores", _I)
_sig("ssa_b200_set_wcorr_gram", _I, _I)
_sig("ssa_b200_wcorr_gram", _I)
_sig("ssa_b200_set_rowmul_tensor_cores", _V, _I)
_sig("ssa_b200_rowmul_tensor_cores", _I)
_sig("ssa_b200_set_context_recycling", _V, _I)
_sig("ssa_b200_context_recycling", _I)
_sig("ssa_b200_device_checks", _I, ctypes.POINTER(ctypes.c_uint), _I)
_sig("ssa_b200_fft_length", _I, _I)


def set_wcorr_tensor_cores(on: bool) -> None:
    """W-correlation Gram on the tensor cores (split TF32, default) or in FP64 on the CUDA cores."""
    _lib.ssa_b200_set_wcorr_tensor_cores(1 if on else 0)


def wcorr_tensor_cores() -> bool:
    return bool(_lib.ssa_b200_wcorr_tensor_cores())


# W-correlation Gram arithmetics (ssa_b200_set_wcorr_gram)
WGRAM_FP64, WGRAM_TF32X3, WGRAM_BF16X3, WGRAM_FP32 = 0, 1, 2, 3
WGRAM_NAMES = {WGRAM_FP64: "fp64", WGRAM_TF32X3: "split-tf32 (tensor cores)",
               WGRAM_BF16X3: "split-bf16 (tensor cores)", WGRAM_FP32: "fp32 (cuda cores)"}


def set_wcorr_gram(mode: int) -> None:
    """The W-correlation Gram's arithmetic for the pipelines: WGRAM_FP64, WGRAM_TF32X3 (default),
    WGRAM_BF16X3 or WGRAM_FP32."""
    if _lib.ssa_b200_set_wcorr_gram(int(mode)) != 0:
        raise ValueError(f"unknown W-correlation Gram mode {mode}")


def wcorr_gram() -> int:
    return int(_lib.ssa_b200_wcorr_gram())


def set_rowmul_tensor_cores(on: bool) -> None:
    """Row products of the randomized pipelines on the tensor cores (three-part TF32 split, six
    products) or in FP32 on the CUDA cores (default)."""
    _lib.ssa_b200_set_rowmul_tensor_cores(1 if on else 0)


def rowmul_tensor_cores() -> bool:
    return bool(_lib.ssa_b200_rowmul_tensor_cores())


def set_context_recycling(on: bool) -> None:
    """Contexts created afterwards recycle streams, pooled device buffers and page-locked staging
    of freed contexts (default) or allocate them afresh."""
    _lib.ssa_b200_set_context_recycling(1 if on else 0)


def context_recycling() -> bool:
    return bool(_lib.ssa_b200_context_recycling())


def device_checks(reset: bool = True) -> List[int]:
    """The kernels' self-check record: [count, kernel, block, code, value] (count 0 = clean)."""
    out = (ctypes.c_uint * 5)()
    _lib.ssa_b200_device_checks(out, 1 if reset else 0)
    return list(out)


PROFILE_KINDS = ("spectrum", "corr", "gram", "chol", "rowmul", "rr", "elem_recon", "wcorr_finish", "group_sum",
                 "recon", "lrf", "wcorr_gram")


def fft_length(N: int) -> int:
    """Real FFT length the uneven batches use for a series of length N (a power of two, or 49152 /
    81920 / 98304 between the cluster powers of two); -1 beyond 131072."""
    return int(_lib.ssa_b200_fft_length(int(N)))


def kernel_launches() -> int:
    """CUDA kernel launches issued by libssa.so in this process."""
    return int(_lib.ssa_b200_kernel_launches())


def _dp(a: np.ndarray):
    return a.ctypes.data_as(c_double_p)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(c_int_p)


class CadzowResult:
    """Result of Cadzow iterations (MKL/py/ssa_wrapper.py:400-413)."""

    def __init__(self, signal: np.ndarray, iterations: int, final_diff: float, converged: bool):
        self.signal = signal
        self.iterations = iterations
        self.final_diff = final_diff
        self.converged = converged

    def __repr__(self):
        return f"CadzowResult(iterations={self.iterations}, final_diff={self.final_diff:.2e}, converged={self.converged})"


def cadzow(x: np.ndarray, L: int, rank: int, max_iter: int = 20, tol: float = 1e-9, alpha: float = 1.0) -> CadzowResult:
    """Cadzow iterations (MKL/py/ssa_wrapper.py:415-489 -> ssa_opt_cadzow)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    N = len(x)
    out = np.zeros(N)
    res = _SSA_CadzowResult()
    if alpha == 1.0:
        ret = _lib.ssa_opt_cadzow(_dp(x), N, L, rank, max_iter, tol, _dp(out), ctypes.byref(res))
    else:
        ret = _lib.ssa_opt_cadzow_weighted(_dp(x), N, L, rank, max_iter, tol, alpha, _dp(out), ctypes.byref(res))
    if ret < 0:
        raise RuntimeError("Cadzow iterations failed")
    return CadzowResult(out, res.iterations, res.final_diff, bool(res.converged))


class _SSA_GapFillResult(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("final_diff", ctypes.c_double), ("converged", ctypes.c_int),
                ("n_gaps", ctypes.c_int)]


_sig("ssa_opt_gapfill", _I, c_double_p, _I, _I, _I, _I, _D, ctypes.POINTER(_SSA_GapFillResult))
_sig("ssa_opt_gapfill_simple", _I, c_double_p, _I, _I, _I, ctypes.POINTER(_SSA_GapFillResult))


class _SSA_ParEstimate(ctypes.Structure):
    _fields_ = [("periods", c_double_p), ("frequencies", c_double_p), ("moduli", c_double_p),
                ("rates", c_double_p), ("n_components", ctypes.c_int)]


_sig("ssa_opt_parestimate", _I, _P, c_int_p, _I, ctypes.POINTER(_SSA_ParEstimate))
_sig("ssa_opt_parestimate_free", _V, ctypes.POINTER(_SSA_ParEstimate))
_sig("ssa_b200_eigvals", _I, _I, c_double_p, c_double_p, c_double_p)


class ParEstimate:
    """ESPRIT result (MKL/py/ssa_wrapper.py:326-413): periods (inf for a trend), frequencies
    (cycles per sample), moduli (1 = undamped) and rates (log modulus) per eigenvalue."""

    def __init__(self, periods, frequencies, moduli, rates):
        self.periods = periods
        self.frequencies = frequencies
        self.moduli = moduli
        self.rates = rates
        self.n_components = len(periods)

    def __repr__(self):
        return f"ParEstimate(n_components={self.n_components})"

    def summary(self) -> str:
        lines = ["ESPRIT Frequency Estimation Results", "=" * 50,
                 f"{'Comp':<6} {'Period':<12} {'Frequency':<12} {'Modulus':<10} {'Rate':<10}", "-" * 50]
        for i in np.argsort(-self.periods):
            p = self.periods[i]
            ps = "Inf (trend)" if np.isinf(p) else f"{p:.2f}"
            lines.append(f"{i:<6} {ps:<12} {self.frequencies[i]:<12.6f} {self.moduli[i]:<10.4f} {self.rates[i]:<10.4f}")
        return "\n".join(lines)

    def get_periodic_components(self, min_period: float = 2.0, max_period: Optional[float] = None,
                                min_modulus: float = 0.9) -> List[int]:
        out = []
        for i in range(self.n_components):
            p, mod = self.periods[i], self.moduli[i]
            if np.isinf(p) or p < min_period or (max_period is not None and p > max_period) or mod < min_modulus:
                continue
            out.append(i)
        return out


def eigvals(A: np.ndarray) -> np.ndarray:
    """Eigenvalues of a real square matrix with the library's host solver (ssa_b200_eigvals)."""
    a = np.ascontiguousarray(A, dtype=np.float64)
    n = a.shape[0]
    wr, wi = np.zeros(n), np.zeros(n)
    if _lib.ssa_b200_eigvals(n, _dp(a), _dp(wr), _dp(wi)) != 0:
        raise RuntimeError("eigenvalues did not converge")
    return wr + 1j * wi


class GapFillResult:
    """Result of gap filling (MKL/py/ssa_wrapper.py:496-509)."""

    def __init__(self, signal: np.ndarray, iterations: int, final_diff: float, converged: bool, n_gaps: int):
        self.signal = signal
        self.iterations = iterations
        self.final_diff = final_diff
        self.converged = converged
        self.n_gaps = n_gaps

    def __repr__(self):
        return (f"GapFillResult(n_gaps={self.n_gaps}, iterations={self.iterations}, "
                f"final_diff={self.final_diff:.2e}, converged={self.converged})")


def gapfill(x: np.ndarray, L: int, rank: int, max_iter: int = 20, tol: float = 1e-6,
            method: str = "iterative") -> GapFillResult:
    """Fill NaN gaps (MKL/py/ssa_wrapper.py:511-590 -> ssa_opt_gapfill / ssa_opt_gapfill_simple):
    "iterative" re-reconstructs the gaps until they settle, "simple" blends a forecast from the
    left and a backcast from the right of every gap."""
    xf = np.ascontiguousarray(np.array(x, dtype=np.float64, copy=True))
    N = len(xf)
    res = _SSA_GapFillResult()
    if method == "iterative":
        ret = _lib.ssa_opt_gapfill(_dp(xf), N, L, rank, max_iter, tol, ctypes.byref(res))
    elif method == "simple":
        ret = _lib.ssa_opt_gapfill_simple(_dp(xf), N, L, rank, ctypes.byref(res))
    else:
        raise ValueError(f"Unknown method: {method}. Use 'iterative' or 'simple'")
    if ret != 0:
        raise RuntimeError(f"Gap filling failed (ret={ret})")
    return GapFillResult(xf, res.iterations, res.final_diff, bool(res.converged), res.n_gaps)


class SSA:
    """Univariate SSA on the GPU (interface of MKL/py/ssa_wrapper.py:600-1202)."""

    def __init__(self, x: np.ndarray, L: int):
        self._ctx = _Opaque1024()
        self._x = np.ascontiguousarray(x, dtype=np.float64)
        self.N = len(self._x)
        self.L = L
        self.K = self.N - L + 1
        self.n_components = 0
        self._decomposed = False
        self._prepared = False
        self._prepared_k = 0
        self._prepared_oversampling = 0
        if _lib.ssa_opt_init(ctypes.byref(self._ctx), _dp(self._x), self.N, L) != 0:
            raise ValueError(f"SSA initialization failed (N={self.N}, L={L})")

    def __del__(self):
        if hasattr(self, "_ctx"):
            _lib.ssa_opt_free(ctypes.byref(self._ctx))

    def prepare(self, max_k: int, oversampling: int = 8) -> "SSA":
        if _lib.ssa_opt_prepare(ctypes.byref(self._ctx), max_k, oversampling) != 0:
            raise RuntimeError(f"prepare() failed (max_k={max_k})")
        self._prepared = True
        self._prepared_k = max_k
        self._prepared_oversampling = oversampling
        return self

    def update_signal(self, new_x: np.ndarray) -> "SSA":
        new_x = np.ascontiguousarray(new_x, dtype=np.float64)
        if len(new_x) != self.N:
            raise ValueError(f"Signal length mismatch: {len(new_x)} vs {self.N}")
        if _lib.ssa_opt_update_signal(ctypes.byref(self._ctx), _dp(new_x)) != 0:
            raise RuntimeError("update_signal() failed")
        self._x = new_x
        return self

    def decompose(self, k: int, method: str = "randomized", **kwargs) -> "SSA":
        """``method`` "randomized" (kwargs: oversampling=8, power_iters=0, omega=None),
        "block" (block_size, max_iter) or "sequential" (max_iter)."""
        if method == "randomized":
            oversampling = kwargs.get("oversampling", 8)
            q = int(kwargs.get("power_iters", 0))
            omega = kwargs.get("omega", None)
            kp = k + oversampling
            if not self._prepared or kp > self._prepared_k + self._prepared_oversampling:
                self.prepare(k, oversampling)
            if q == 0 and omega is None:
                ret = _lib.ssa_opt_decompose_randomized(ctypes.byref(self._ctx), k, oversampling)
            else:
                om = None
                if omega is not None:
                    om = np.asfortranarray(omega, dtype=np.float64)
                    if om.shape[0] != self.K:
                        raise ValueError(f"omega must have K={self.K} rows")
                    om = np.ascontiguousarray(om.T)  # column-major K x kp as flat memory
                ret = _lib.ssa_opt_decompose_randomized_ex(ctypes.byref(self._ctx), k, oversampling, q,
                                                            _dp(om) if om is not None else None)
        elif method == "block":
            block_size = kwargs.get("block_size", min(k, 32))
            max_iter = kwargs.get("max_iter", 100)
            v0 = kwargs.get("v0", None)
            if v0 is None:
                ret = _lib.ssa_opt_decompose_block(ctypes.byref(self._ctx), k, block_size, max_iter)
            else:
                v = np.ascontiguousarray(np.asarray(v0, dtype=np.float64).T)  # K x k column-major
                ret = _lib.ssa_opt_decompose_block_ex(ctypes.byref(self._ctx), k, block_size, max_iter, _dp(v))
        elif method == "sequential":
            ret = _lib.ssa_opt_decompose(ctypes.byref(self._ctx), k, kwargs.get("max_iter", 100))
        else:
            raise ValueError(f"Unknown method: {method}")
        if ret != 0:
            raise RuntimeError(f"Decomposition failed (method={method}, k={k})")
        self.n_components = min(k, min(self.L, self.K))
        self._decomposed = True
        return self

    def _need(self):
        if not self._decomposed:
            raise RuntimeError("Call decompose() first")

    @property
    def singular_values(self) -> np.ndarray:
        self._need()
        out = np.zeros(self.n_components)
        n = _lib.ssa_opt_get_singular_values(ctypes.byref(self._ctx), _dp(out), self.n_components)
        return out[:n]

    @property
    def eigenvalues(self) -> np.ndarray:
        self._need()
        out = np.zeros(self.n_components)
        n = _lib.ssa_opt_get_eigenvalues(ctypes.byref(self._ctx), _dp(out), self.n_components)
        return out[:n]

    @property
    def total_variance(self) -> float:
        self._need()
        return _lib.ssa_opt_get_total_variance(ctypes.byref(self._ctx))

    def reconstruct(self, group: List[int]) -> np.ndarray:
        self._need()
        out = np.zeros(self.N)
        g = np.ascontiguousarray(group, dtype=np.int32)
        if _lib.ssa_opt_reconstruct(ctypes.byref(self._ctx), _ip(g), len(group), _dp(out)) != 0:
            raise RuntimeError("Reconstruction failed")
        return out

    def cache_ffts(self) -> "SSA":
        if _lib.ssa_opt_cache_ffts(ctypes.byref(self._ctx)) != 0:
            raise RuntimeError("cache_ffts failed")
        return self

    def forecast(self, group: List[int], n_forecast: int) -> np.ndarray:
        self._need()
        out = np.zeros(n_forecast)
        g = np.ascontiguousarray(group, dtype=np.int32)
        if _lib.ssa_opt_forecast(ctypes.byref(self._ctx), _ip(g), len(group), n_forecast, _dp(out)) != 0:
            raise RuntimeError("Forecast failed (verticality >= 1?)")
        return out

    def forecast_full(self, group: List[int], n_forecast: int) -> np.ndarray:
        self._need()
        out = np.zeros(self.N + n_forecast)
        g = np.ascontiguousarray(group, dtype=np.int32)
        if _lib.ssa_opt_forecast_full(ctypes.byref(self._ctx), _ip(g), len(group), n_forecast, _dp(out)) != 0:
            raise RuntimeError("Forecast failed")
        return out

    def vforecast(self, group: List[int], n_forecast: int) -> np.ndarray:
        """V-forecast (ssa_opt_vforecast): the projection recurrence, equal to the LRF forecast."""
        self._need()
        out = np.zeros(n_forecast)
        g = np.ascontiguousarray(group, dtype=np.int32)
        if _lib.ssa_opt_vforecast(ctypes.byref(self._ctx), _ip(g), len(group), n_forecast, _dp(out)) != 0:
            raise RuntimeError("V-forecast failed (verticality >= 1?)")
        return out

    def vforecast_full(self, group: List[int], n_forecast: int) -> np.ndarray:
        """Reconstruction of the group followed by its V-forecast (N + n_forecast values)."""
        self._need()
        out = np.zeros(self.N + n_forecast)
        g = np.ascontiguousarray(group, dtype=np.int32)
        if _lib.ssa_opt_vforecast_full(ctypes.byref(self._ctx), _ip(g), len(group), n_forecast, _dp(out)) != 0:
            raise RuntimeError("V-forecast failed")
        return out

    def vforecast_fast(self, group: List[int], base_signal: np.ndarray, n_forecast: int) -> np.ndarray:
        """V-forecast continuing from the last L - 1 values of base_signal."""
        self._need()
        base = np.ascontiguousarray(base_signal, dtype=np.float64)
        out = np.zeros(n_forecast)
        g = np.ascontiguousarray(group, dtype=np.int32)
        if _lib.ssa_opt_vforecast_fast(ctypes.byref(self._ctx), _ip(g), len(group), _dp(base), len(base),
                                       n_forecast, _dp(out)) != 0:
            raise RuntimeError("V-forecast failed")
        return out

    def lrf(self, group: List[int]) -> Tuple[np.ndarray, float]:
        """LRF coefficients R (L - 1) and verticality nu^2 (ssa_opt_compute_lrf)."""
        self._need()
        g = np.ascontiguousarray(group, dtype=np.int32)
        lrf = _SSA_LRF()
        if _lib.ssa_opt_compute_lrf(ctypes.byref(self._ctx), _ip(g), len(group), ctypes.byref(lrf)) != 0:
            raise RuntimeError("compute_lrf failed")
        R = np.ctypeslib.as_array(lrf.R, shape=(self.L - 1,)).copy()
        v = lrf.verticality
        _lib.ssa_opt_lrf_free(ctypes.byref(lrf))
        return R, v

    def get_trend(self) -> np.ndarray:
        self._need()
        out = np.zeros(self.N)
        if _lib.ssa_opt_get_trend(ctypes.byref(self._ctx), _dp(out)) != 0:
            raise RuntimeError("get_trend failed")
        return out

    def get_noise(self, noise_start: int) -> np.ndarray:
        self._need()
        out = np.zeros(self.N)
        if _lib.ssa_opt_get_noise(ctypes.byref(self._ctx), noise_start, _dp(out)) != 0:
            raise RuntimeError("get_noise failed")
        return out

    def cadzow(self, rank: int, max_iter: int = 20, tol: float = 1e-9, alpha: float = 1.0) -> CadzowResult:
        return cadzow(self._x, self.L, rank, max_iter, tol, alpha)

    def cadzow_inplace(self, rank: int, max_iter: int = 20, tol: float = 1e-9) -> CadzowResult:
        """In-place Cadzow on this context (ssa_opt_cadzow_inplace): the context's signal becomes
        the iterate and its decomposition the last one; ``signal`` is its rank-``rank``
        reconstruction."""
        res = _SSA_CadzowResult()
        ret = _lib.ssa_opt_cadzow_inplace(ctypes.byref(self._ctx), rank, max_iter, tol, ctypes.byref(res))
        if ret < 0:
            raise RuntimeError("in-place Cadzow iterations failed")
        self._decomposed = True
        self.n_components = int(_lib.ssa_opt_copy_factors(ctypes.byref(self._ctx), None, None))
        return CadzowResult(self.reconstruct(list(range(rank))), res.iterations, res.final_diff,
                            bool(res.converged))

    def wcorr_matrix(self) -> np.ndarray:
        self._need()
        k = self.n_components
        W = np.zeros((k, k))
        if _lib.ssa_opt_wcorr_matrix(ctypes.byref(self._ctx), _dp(W)) != 0:
            raise RuntimeError("wcorr_matrix failed")
        return W

    def wcorr(self, i: int, j: int) -> float:
        self._need()
        return _lib.ssa_opt_wcorr_pair(ctypes.byref(self._ctx), i, j)

    def variance_explained(self, start: int = 0, end: int = -1) -> float:
        self._need()
        return _lib.ssa_opt_variance_explained(ctypes.byref(self._ctx), start, end)

    def component_stats(self) -> dict:
        """ssa_opt_component_stats: sigma, log sigma, neighbour drop ratios, cumulative variance,
        log-spectrum curvature, suggested signal rank and its drop ratio."""
        self._need()
        st = _ComponentStats()
        if _lib.ssa_opt_component_stats(ctypes.byref(self._ctx), ctypes.byref(st)) != 0:
            raise RuntimeError("component_stats failed")
        n = st.n
        try:
            out = {"singular_values": np.ctypeslib.as_array(st.singular_values, (n,)).copy(),
                   "log_sv": np.ctypeslib.as_array(st.log_sv, (n,)).copy(),
                   "gaps": np.ctypeslib.as_array(st.gaps, (n - 1,)).copy(),
                   "cumulative_var": np.ctypeslib.as_array(st.cumulative_var, (n,)).copy(),
                   "second_diff": np.ctypeslib.as_array(st.second_diff, (n,)).copy(),
                   "suggested_signal": int(st.suggested_signal), "gap_threshold": float(st.gap_threshold)}
        finally:
            _lib.ssa_opt_component_stats_free(ctypes.byref(st))
        return out

    def find_periodic_pairs(self, max_pairs: int = 10, sv_tol: float = 0.1,
                            wcorr_thresh: float = 0.5) -> List[Tuple[int, int]]:
        self._need()
        pairs = np.zeros(2 * max_pairs, dtype=np.int32)
        n = _lib.ssa_opt_find_periodic_pairs(ctypes.byref(self._ctx), _ip(pairs), max_pairs, sv_tol, wcorr_thresh)
        return [(int(pairs[2 * i]), int(pairs[2 * i + 1])) for i in range(n)]

    def hankel_matvec(self, v: np.ndarray) -> np.ndarray:
        """y = H v on the device (invalidates a previous decomposition of this object)."""
        v = np.ascontiguousarray(v, dtype=np.float64)
        y = np.zeros(self.L)
        if _lib.ssa_opt_hankel_matvec_dev(ctypes.byref(self._ctx), _dp(v), _dp(y)) != 0:
            raise RuntimeError("hankel_matvec failed")
        self._decomposed = False
        return y

    def hankel_matvec_T(self, u: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64)
        z = np.zeros(self.K)
        if _lib.ssa_opt_hankel_matvec_T_dev(ctypes.byref(self._ctx), _dp(u), _dp(z)) != 0:
            raise RuntimeError("hankel_matvec_T failed")
        self._decomposed = False
        return z

    # factor access (host mirrors of the SSA_Opt fields U, V)
    def factors(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(U L x k, V K x k, sigma k) copied from the context's host fields."""
        self._need()
        k = self.n_components
        U = np.zeros((k, self.L))
        V = np.zeros((k, self.K))
        if _lib.ssa_opt_copy_factors(ctypes.byref(self._ctx), _dp(U), _dp(V)) != k:
            raise RuntimeError("copy_factors failed")
        return U.T.copy(), V.T.copy(), self.singular_values

    def extend(self, additional_k: int, max_iter: int = 100) -> "SSA":
        """Add components to the current decomposition by deflated one-column power iterations
        (ssa_opt_extend, MKL/ssa_opt.h:1935-2056); all are then re-sorted by sigma."""
        self._need()
        if _lib.ssa_opt_extend(ctypes.byref(self._ctx), additional_k, max_iter) != 0:
            raise RuntimeError("extend failed")
        self.n_components = int(_lib.ssa_opt_copy_factors(ctypes.byref(self._ctx), None, None))
        return self

    def parestimate(self, group: Optional[List[int]] = None) -> "ParEstimate":
        """ESPRIT periods / frequencies / moduli / rates of the selected components (all when
        group is None), MKL/py/ssa_wrapper.py:1061-1130 -> ssa_opt_parestimate."""
        self._need()
        res = _SSA_ParEstimate()
        if group is not None and len(group) > 0:
            g = np.ascontiguousarray(group, dtype=np.int32)
            ret = _lib.ssa_opt_parestimate(ctypes.byref(self._ctx), _ip(g), len(g), ctypes.byref(res))
        else:
            ret = _lib.ssa_opt_parestimate(ctypes.byref(self._ctx), None, 0, ctypes.byref(res))
        if ret != 0:
            raise RuntimeError("parestimate failed")
        n = res.n_components
        arrs = [np.ctypeslib.as_array(getattr(res, f), shape=(n,)).copy()
                for f in ("periods", "frequencies", "moduli", "rates")]
        _lib.ssa_opt_parestimate_free(ctypes.byref(res))
        return ParEstimate(*arrs)


class MSSA:
    """Multivariate SSA on the GPU (interface of MKL/py/ssa_wrapper.py:1208-1371)."""

    def __init__(self, X: np.ndarray, L: int):
        self._ctx = _Opaque1024()
        self._X = np.ascontiguousarray(X, dtype=np.float64)
        if self._X.ndim != 2:
            raise ValueError("X must be 2D array of shape (M, N)")
        self.M, self.N = self._X.shape
        self.L = L
        self.K = self.N - L + 1
        self.n_components = 0
        self._decomposed = False
        if _lib.mssa_opt_init(ctypes.byref(self._ctx), _dp(self._X), self.M, self.N, L) != 0:
            raise ValueError(f"MSSA initialization failed (M={self.M}, N={self.N}, L={L})")

    def __del__(self):
        if hasattr(self, "_ctx"):
            _lib.mssa_opt_free(ctypes.byref(self._ctx))

    def decompose(self, k: int, oversampling: int = 8, power_iters: int = 0,
                  omega: Optional[np.ndarray] = None) -> "MSSA":
        if power_iters == 0 and omega is None:
            ret = _lib.mssa_opt_decompose(ctypes.byref(self._ctx), k, oversampling)
        else:
            om = None
            if omega is not None:
                om = np.ascontiguousarray(np.asarray(omega, dtype=np.float64).T)
            ret = _lib.mssa_opt_decompose_ex(ctypes.byref(self._ctx), k, oversampling, power_iters,
                                             _dp(om) if om is not None else None)
        if ret != 0:
            raise RuntimeError(f"MSSA decomposition failed (k={k})")
        self.n_components = int(_lib.mssa_opt_copy_factors(ctypes.byref(self._ctx), None, None, None))
        self._decomposed = True
        return self

    def factors(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(U (M L x k), V (K x k), sigma (k)) of the last decomposition."""
        if not self._decomposed:
            raise RuntimeError("Call decompose() first")
        k = self.n_components
        U = np.zeros((k, self.M * self.L))
        V = np.zeros((k, self.K))
        s = np.zeros(k)
        if _lib.mssa_opt_copy_factors(ctypes.byref(self._ctx), _dp(U), _dp(V), _dp(s)) != k:
            raise RuntimeError("copy_factors failed")
        return U.T.copy(), V.T.copy(), s

    @property
    def singular_values(self) -> np.ndarray:
        return self.factors()[2]

    def reconstruct(self, series_idx: int, group: List[int]) -> np.ndarray:
        if not self._decomposed:
            raise RuntimeError("Call decompose() first")
        out = np.zeros(self.N)
        g = np.ascontiguousarray(group, dtype=np.int32)
        if _lib.mssa_opt_reconstruct(ctypes.byref(self._ctx), series_idx, _ip(g), len(group), _dp(out)) != 0:
            raise RuntimeError("Reconstruction failed")
        return out

    def reconstruct_all(self, group: List[int]) -> np.ndarray:
        if not self._decomposed:
            raise RuntimeError("Call decompose() first")
        out = np.zeros((self.M, self.N))
        g = np.ascontiguousarray(group, dtype=np.int32)
        if _lib.mssa_opt_reconstruct_all(ctypes.byref(self._ctx), _ip(g), len(group), _dp(out)) != 0:
            raise RuntimeError("Reconstruction failed")
        return out

    def series_contributions(self) -> np.ndarray:
        if not self._decomposed:
            raise RuntimeError("Call decompose() first")
        c = np.zeros((self.M, self.n_components))
        if _lib.mssa_opt_series_contributions(ctypes.byref(self._ctx), _dp(c)) != 0:
            raise RuntimeError("series_contributions failed")
        return c

    def variance_explained(self, start: int = 0, end: int = -1) -> float:
        if not self._decomposed:
            raise RuntimeError("Call decompose() first")
        return _lib.mssa_opt_variance_explained(ctypes.byref(self._ctx), start, end)


class SSABatch:
    """Batched pipeline for up to ``max_series`` series of length N: decomposition, all k
    elementary reconstructions, W-correlation and the sums of ``groups`` (ssa_batch_* C ABI)."""

    def __init__(self, max_series: int, N: int, L: int, k: int, oversampling: int = 10, power_iters: int = 2,
                 groups: Sequence[Sequence[int]] = ((0,), (1, 2))):
        self.max_series, self.N, self.L = max_series, N, L
        K = N - L + 1
        kp = min(k + oversampling, L, K)
        self.k = min(k, kp)
        self.groups = [list(g) for g in groups]
        idx = np.ascontiguousarray([i for g in self.groups for i in g] or [0], dtype=np.int32)
        sizes = np.ascontiguousarray([len(g) for g in self.groups] or [0], dtype=np.int32)
        self._h = ctypes.c_void_p()
        if _lib.ssa_batch_create(ctypes.byref(self._h), max_series, N, L, k, oversampling, power_iters,
                                 _ip(idx), _ip(sizes), len(self.groups)) != 0:
            raise ValueError("ssa_batch_create failed")
        self._keep = (idx, sizes)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.ssa_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def run(self, X: np.ndarray, seed: int = 0):
        """Host-to-host run. Returns (sigma B x k, W B x k x k, groups B x n_groups x N)."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        B = X.shape[0]
        sigma = np.zeros((B, self.k))
        W = np.zeros((B, self.k, self.k))
        G = np.zeros((B, len(self.groups), self.N))
        if _lib.ssa_batch_run(self._h, _dp(X), B, seed, _dp(sigma), _dp(W), _dp(G) if self.groups else None) != 0:
            raise RuntimeError("ssa_batch_run failed")
        return sigma, W, G

    def run_device(self, d_x_ptr: int, B: int, seed: int = 0) -> None:
        """Enqueue a run on device-resident input (B x N doubles at device address d_x_ptr)."""
        if _lib.ssa_batch_run_device(self._h, ctypes.c_void_p(d_x_ptr), B, seed) != 0:
            raise RuntimeError("ssa_batch_run_device failed")

    def run_host_ptrs(self, x_ptr: int, B: int, seed: int, sigma_ptr: int, W_ptr: int, groups_ptr: int) -> None:
        """Host-to-host run on caller-owned (ideally pinned) buffers given by address."""
        vp = lambda a: ctypes.cast(ctypes.c_void_p(a), c_double_p) if a else None  # noqa: E731
        if _lib.ssa_batch_run(self._h, vp(x_ptr), B, seed, vp(sigma_ptr), vp(W_ptr), vp(groups_ptr)) != 0:
            raise RuntimeError("ssa_batch_run failed")

    def sync(self) -> None:
        if _lib.ssa_batch_sync(self._h) != 0:
            raise RuntimeError("a series of the batch failed")

    def status(self, n: int) -> np.ndarray:
        """Status words of the first n series of the last run (0 = ok)."""
        st = np.zeros(n, dtype=np.int32)
        if _lib.ssa_batch_status(self._h, _ip(st), n) != 0:
            raise RuntimeError("ssa_batch_status failed")
        return st

    def set_profiling(self, on: bool) -> None:
        if _lib.ssa_batch_set_profiling(self._h, 1 if on else 0) != 0:
            raise RuntimeError("ssa_batch_set_profiling failed")

    def profile(self) -> dict:
        """{kind: (milliseconds, launches)} accumulated since profiling was switched on."""
        ms = (ctypes.c_double * len(PROFILE_KINDS))()
        n = (ctypes.c_longlong * len(PROFILE_KINDS))()
        if _lib.ssa_batch_profile(self._h, ms, n, len(PROFILE_KINDS)) < 0:
            raise RuntimeError("ssa_batch_profile failed")
        return {k: (ms[i], int(n[i])) for i, k in enumerate(PROFILE_KINDS)}

    def device_results(self) -> dict:
        r = _BatchResults()
        if _lib.ssa_batch_device_results(self._h, ctypes.byref(r)) != 0:
            raise RuntimeError("ssa_batch_device_results failed")
        return {"sigma": r.sigma, "W": r.W, "groups": r.groups, "recon": r.recon, "ld_recon": r.ld_recon,
                "status": r.status, "stream": r.stream}


_sig("ssa_rbatch_create", _I, ctypes.POINTER(ctypes.c_void_p), _I, _I, c_int_p, c_int_p, _I)
_sig("ssa_rbatch_destroy", _V, ctypes.c_void_p)
_sig("ssa_rbatch_run", _I, ctypes.c_void_p, _I, c_int_p, c_int_p, c_int_p, c_double_p, ctypes.c_uint64,
     c_double_p, c_double_p, c_double_p)
_sig("ssa_rbatch_run_device", _I, ctypes.c_void_p, _I, c_int_p, c_int_p, c_int_p, ctypes.c_void_p, ctypes.c_uint64)
_sig("ssa_rbatch_run_ex", _I, ctypes.c_void_p, _I, c_int_p, c_int_p, c_int_p, c_double_p, ctypes.c_uint64,
     c_double_p, c_double_p, c_double_p, ctypes.c_void_p)
_sig("ssa_rbatch_run_device_ex", _I, ctypes.c_void_p, _I, c_int_p, c_int_p, c_int_p, ctypes.c_void_p,
     ctypes.c_uint64, ctypes.c_void_p)
_sig("ssa_rbatch_sync", _I, ctypes.c_void_p)
_sig("ssa_rbatch_layout", _I, ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t))
_sig("ssa_rbatch_device_results", _I, ctypes.c_void_p, ctypes.POINTER(_BatchResults))
_sig("ssa_rbatch_set_profiling", _I, ctypes.c_void_p, _I)
_sig("ssa_rbatch_profile", _I, ctypes.c_void_p, c_double_p, ctypes.POINTER(ctypes.c_longlong), _I)


def set_multi_length(on: bool) -> None:
    """Series of real FFT length 512..16384 in one persistent multi-length sweep launch (default)
    or one bucket per length."""
    _lib.ssa_b200_set_multi_length(1 if on else 0)


def multi_length() -> bool:
    return bool(_lib.ssa_b200_multi_length())


class SSARaggedBatch:
    """Uneven batch (ssa_rbatch_* C ABI): series of different N, L and k through decomposition,
    all elementary reconstructions, W-correlation and the sums of ``groups`` in one pass, one
    launch per stage per FFT-length bucket."""

    def __init__(self, oversampling: int = 10, power_iters: int = 2,
                 groups: Sequence[Sequence[int]] = ((0,), (1, 2))):
        self.p, self.q = oversampling, power_iters
        self.groups = [list(g) for g in groups]
        idx = np.ascontiguousarray([i for g in self.groups for i in g] or [0], dtype=np.int32)
        sizes = np.ascontiguousarray([len(g) for g in self.groups] or [0], dtype=np.int32)
        self._h = ctypes.c_void_p()
        if _lib.ssa_rbatch_create(ctypes.byref(self._h), oversampling, power_iters, _ip(idx), _ip(sizes),
                                  len(self.groups)) != 0:
            raise ValueError("ssa_rbatch_create failed")
        self._keep = (idx, sizes)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.ssa_rbatch_destroy(self._h)
            self._h = ctypes.c_void_p()

    @staticmethod
    def _dims(N, L, k):
        N = np.ascontiguousarray(N, dtype=np.int32)
        L = np.ascontiguousarray(L, dtype=np.int32)
        k = np.ascontiguousarray(k, dtype=np.int32)
        if not (len(N) == len(L) == len(k)):
            raise ValueError("N, L and k must have one entry per series")
        return N, L, k

    @staticmethod
    def effective_k(N, L, k) -> np.ndarray:
        """Components per series: min(k, L, N - L + 1) (at least 1 for the output layout)."""
        N, L, k = (np.asarray(a, dtype=np.int64) for a in (N, L, k))
        return np.maximum(np.minimum(k, np.minimum(L, N - L + 1)), 1)

    @staticmethod
    def _mask(want_w, B):
        """Per-series W-correlation flags as a uint8 array (None = W for every series)."""
        if want_w is None:
            return None, None
        m = np.ascontiguousarray(np.asarray(want_w, dtype=bool).astype(np.uint8))
        if m.shape != (B,):
            raise ValueError("want_w must have one entry per series")
        return m, ctypes.c_void_p(m.ctypes.data)

    def run(self, series: Sequence[np.ndarray], L: Sequence[int], k: Sequence[int], seed: int = 0, want_w=None):
        """Host-to-host run. Returns per-series lists (sigma, W, groups). With want_w (one flag per
        series) only the flagged series get their W-correlation (the others' W is zero) and the
        others compute only the elementary reconstructions their groups use."""
        Na, La, ka = self._dims([len(x) for x in series], L, k)
        m, mp = self._mask(want_w, len(Na))
        x = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.float64) for s in series]))
        ke = self.effective_k(Na, La, ka)
        sig = np.zeros(int(ke.sum()))
        W = np.zeros(int((ke * ke).sum()))
        G = np.zeros(max(1, len(self.groups) * int(Na.sum())))
        if _lib.ssa_rbatch_run_ex(self._h, len(Na), _ip(Na), _ip(La), _ip(ka), _dp(x), seed, _dp(sig), _dp(W),
                                  _dp(G) if self.groups else None, mp) != 0:
            raise RuntimeError("ssa_rbatch_run failed")
        return self._unpack(Na, ke, sig, W, G)

    def _unpack(self, Na, ke, sig, W, G):
        out_s, out_w, out_g = [], [], []
        o_s = o_w = o_g = 0
        ng = len(self.groups)
        for n, kk in zip(Na.tolist(), ke.tolist()):
            out_s.append(sig[o_s:o_s + kk])
            out_w.append(W[o_w:o_w + kk * kk].reshape(kk, kk))
            out_g.append(G[o_g:o_g + ng * n].reshape(ng, n))
            o_s += kk
            o_w += kk * kk
            o_g += ng * n
        return out_s, out_w, out_g

    def run_device(self, d_x_ptr: int, N, L, k, seed: int = 0, want_w=None) -> None:
        """Enqueue a run on device-resident packed input (sum N doubles at d_x_ptr); want_w as in
        run()."""
        Na, La, ka = self._dims(N, L, k)
        m, mp = self._mask(want_w, len(Na))
        if _lib.ssa_rbatch_run_device_ex(self._h, len(Na), _ip(Na), _ip(La), _ip(ka), ctypes.c_void_p(d_x_ptr),
                                         seed, mp) != 0:
            raise RuntimeError("ssa_rbatch_run_device failed")

    def run_host_ptrs(self, N, L, k, x_ptr: int, seed: int, sigma_ptr: int, W_ptr: int, groups_ptr: int) -> None:
        """Host-to-host run on caller-owned (ideally pinned) packed buffers given by address."""
        Na, La, ka = self._dims(N, L, k)
        vp = lambda a: ctypes.cast(ctypes.c_void_p(a), c_double_p) if a else None  # noqa: E731
        if _lib.ssa_rbatch_run(self._h, len(Na), _ip(Na), _ip(La), _ip(ka), vp(x_ptr), seed, vp(sigma_ptr),
                               vp(W_ptr), vp(groups_ptr)) != 0:
            raise RuntimeError("ssa_rbatch_run failed")

    def sync(self) -> None:
        if _lib.ssa_rbatch_sync(self._h) != 0:
            raise RuntimeError("a series of the uneven batch failed")

    def set_profiling(self, on, serialize: bool = False) -> None:
        """Per-kernel CUDA-event times; with serialize=True the FFT-length buckets run one after
        another so that each launch's interval is its own."""
        mode = (2 if serialize else 1) if on else 0
        if _lib.ssa_rbatch_set_profiling(self._h, mode) != 0:
            raise RuntimeError("ssa_rbatch_set_profiling failed")

    def profile(self) -> dict:
        """{kind: (milliseconds summed over buckets, launches)} since profiling was switched on."""
        ms = (ctypes.c_double * len(PROFILE_KINDS))()
        n = (ctypes.c_longlong * len(PROFILE_KINDS))()
        if _lib.ssa_rbatch_profile(self._h, ms, n, len(PROFILE_KINDS)) < 0:
            raise RuntimeError("ssa_rbatch_profile failed")
        return {kk: (ms[i], int(n[i])) for i, kk in enumerate(PROFILE_KINDS)}

    def device_results(self) -> dict:
        r = _BatchResults()
        if _lib.ssa_rbatch_device_results(self._h, ctypes.byref(r)) != 0:
            raise RuntimeError("ssa_rbatch_device_results failed")
        return {"sigma": r.sigma, "W": r.W, "groups": r.groups, "status": r.status, "stream": r.stream}

    def set_graphs(self, on: bool) -> None:
        """CUDA-graph capture and replay of runs with a repeated launch signature (default on)."""
        _lib.ssa_rbatch_set_graphs(self._h, 1 if on else 0)

    def graph_stats(self) -> dict:
        c, r = ctypes.c_longlong(), ctypes.c_longlong()
        _lib.ssa_rbatch_graph_stats(self._h, ctypes.byref(c), ctypes.byref(r))
        return {"captures": c.value, "replays": r.value}

    def series_result(self, s: int, N: int, L: int, k: int, factors: bool = False) -> dict:
        """Outputs of series s of the last run (waits for it): sigma, W, groups and, with
        factors=True, U (L x k') and V (K x k')."""
        ke = int(self.effective_k([N], [L], [k])[0])
        K = N - L + 1
        sig, W = np.zeros(ke), np.zeros((ke, ke))
        G = np.zeros((max(1, len(self.groups)), N))
        U = np.zeros((ke, L)) if factors else None
        V = np.zeros((ke, K)) if factors else None
        n = _lib.ssa_rbatch_series_result(self._h, s, _dp(sig), _dp(W), _dp(G) if self.groups else None,
                                          _dp(U) if factors else None, _dp(V) if factors else None)
        if n != ke:
            raise RuntimeError("ssa_rbatch_series_result failed")
        out = {"sigma": sig, "W": W, "groups": G[:len(self.groups)]}
        if factors:
            out["U"], out["V"] = U.T, V.T
        return out


_sig("ssa_mbatch_create", _I, ctypes.POINTER(ctypes.c_void_p), _I, _I, _I, _I, _I, _I, _I)
_sig("ssa_mbatch_destroy", _V, ctypes.c_void_p)
_sig("ssa_mbatch_run_device", _I, ctypes.c_void_p, ctypes.c_void_p, _I, ctypes.c_uint64, ctypes.c_void_p,
     ctypes.c_void_p)
_sig("ssa_mbatch_sync", _I, ctypes.c_void_p)
_sig("ssa_mbatch_diffs", _I, ctypes.c_void_p, _I, c_double_p)
_sig("ssa_mbatch_run", _I, ctypes.c_void_p, c_double_p, _I, ctypes.c_uint64, c_double_p, c_double_p, c_double_p)
_sig("ssa_mbatch_dims", _I, ctypes.c_void_p, c_int_p, c_int_p)
_sig("ssa_mbatch_stream", ctypes.c_void_p, ctypes.c_void_p)


class SSAMultiBatch:
    """Batched multichannel SSA with Cadzow iterations (ssa_mbatch_* C ABI): I instances of M
    channels of length N, block power of every stacked operator and `iters` multivariate Cadzow
    iterations, all instances together."""

    def __init__(self, instances: int, M: int, N: int, L: int, k: int, oversampling: int = 10,
                 power_iters: int = 2):
        self.I, self.M, self.N, self.L = instances, M, N, L
        self._h = ctypes.c_void_p()
        if _lib.ssa_mbatch_create(ctypes.byref(self._h), instances, M, N, L, k, oversampling, power_iters) != 0:
            raise ValueError("ssa_mbatch_create failed")
        kk, kp = ctypes.c_int(), ctypes.c_int()
        _lib.ssa_mbatch_dims(self._h, ctypes.byref(kk), ctypes.byref(kp))
        self.k, self.kp = kk.value, kp.value

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.ssa_mbatch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def run(self, X: np.ndarray, iters: int, seed: int = 0):
        """X: (I, M, N). Returns (channels after the iterations (I, M, N), sigma (I, k), relative
        change per iteration (I, iters))."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        if X.shape != (self.I, self.M, self.N):
            raise ValueError(f"X must have shape {(self.I, self.M, self.N)}")
        out = np.zeros_like(X)
        sig = np.zeros((self.I, self.k))
        diff = np.zeros((self.I, iters))
        if _lib.ssa_mbatch_run(self._h, _dp(X), iters, seed, _dp(out), _dp(sig), _dp(diff)) != 0:
            raise RuntimeError("ssa_mbatch_run failed")
        return out, sig, diff

    def run_device(self, d_x_ptr: int, iters: int, seed: int = 0, d_out_ptr: int = 0, d_sigma_ptr: int = 0) -> None:
        if _lib.ssa_mbatch_run_device(self._h, ctypes.c_void_p(d_x_ptr), iters, seed,
                                      ctypes.c_void_p(d_out_ptr or None), ctypes.c_void_p(d_sigma_ptr or None)) != 0:
            raise RuntimeError("ssa_mbatch_run_device failed")

    def sync(self) -> None:
        if _lib.ssa_mbatch_sync(self._h) != 0:
            raise RuntimeError("an instance of the multichannel batch failed")

    def diffs(self, iters: int) -> np.ndarray:
        d = np.zeros((self.I, iters))
        if _lib.ssa_mbatch_diffs(self._h, iters, _dp(d)) != 0:
            raise RuntimeError("ssa_mbatch_diffs failed")
        return d

    @property
    def stream(self) -> int:
        return int(_lib.ssa_mbatch_stream(self._h) or 0)


class _Request(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("series_id", ctypes.c_int), ("N", ctypes.c_int), ("L", ctypes.c_int),
                ("k", ctypes.c_int), ("h", ctypes.c_int), ("x", c_double_p), ("seed", ctypes.c_uint64),
                ("sigma", c_double_p), ("groups", c_double_p), ("W", c_double_p), ("forecast", c_double_p),
                ("status", ctypes.c_int), ("k_out", ctypes.c_int), ("t_arrival", ctypes.c_double),
                ("t_done", ctypes.c_double), ("priv", ctypes.c_void_p),
                ("group", c_int_p), ("n_group", ctypes.c_int), ("rank", ctypes.c_int), ("max_iter", ctypes.c_int),
                ("tol", ctypes.c_double), ("out", c_double_p), ("iterations", ctypes.c_int),
                ("final_diff", ctypes.c_double)]


class _ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_longlong) for n in ("submitted", "completed", "failed", "batches", "decompositions",
                                                  "max_batch", "forecast_batches", "forecasts", "evictions",
                                                  "not_resident")] + \
               [(n, ctypes.c_size_t) for n in ("resident_bytes", "resident_budget", "batch_budget")] + \
               [(n, ctypes.c_double) for n in ("host_launch_s", "host_finish_s", "host_launch_max_s")] + \
               [(n, ctypes.c_longlong) for n in ("followup_batches", "followups", "cadzow_requests",
                                                  "cadzow_iterations")]


_sig("ssa_b200_set_multi_length", _V, _I)
_sig("ssa_b200_multi_length", _I)
_sig("ssa_rbatch_set_graphs", _I, ctypes.c_void_p, _I)
_sig("ssa_rbatch_graph_stats", _I, ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong))
_sig("ssa_rbatch_series_result", _I, ctypes.c_void_p, _I, c_double_p, c_double_p, c_double_p, c_double_p,
     c_double_p)
_sig("ssa_server_create", _I, ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t, _I, _I, _I, _I)
_sig("ssa_server_destroy", _V, ctypes.c_void_p)
_sig("ssa_server_submit", _I, ctypes.c_void_p, ctypes.POINTER(_Request))
_sig("ssa_server_drain", _I, ctypes.c_void_p)
_sig("ssa_server_replay", _I, ctypes.c_void_p, ctypes.POINTER(_Request), c_double_p, _I)
_sig("ssa_server_stats_get", _I, ctypes.c_void_p, ctypes.POINTER(_ServerStats))
_sig("ssa_server_now", _D)
_sig("ssa_host_alloc", ctypes.c_void_p, ctypes.c_size_t)
_sig("ssa_host_free", _V, ctypes.c_void_p)


class _PinnedPool:
    """Page-locked host arrays (ssa_host_alloc), freed with the pool."""

    def __init__(self):
        self._ptrs = []

    def array(self, shape, src: Optional[np.ndarray] = None) -> np.ndarray:
        n = int(np.prod(shape))
        p = _lib.ssa_host_alloc(max(1, n) * 8)
        if not p:
            raise MemoryError("ssa_host_alloc failed")
        self._ptrs.append(p)
        a = np.ctypeslib.as_array(ctypes.cast(p, c_double_p), shape=(max(1, n),))[:n].reshape(shape)
        if src is not None:
            a[...] = src
        else:
            a[...] = 0.0
        return a

    def __del__(self):
        for p in self._ptrs:
            _lib.ssa_host_free(p)
        self._ptrs = []

REQ_DECOMPOSE_RECON, REQ_DECOMPOSE_WCORR, REQ_FORECAST, REQ_RECONSTRUCT, REQ_CADZOW = 0, 1, 2, 3, 4


class Requests:
    """A block of requests for SSAServer (ssa_request array) with their host buffers.

    ``add_decompose(x, L, k, series_id, seed, wcorr=False)`` and ``add_forecast(series_id, h)``
    append requests; after the server has completed them, ``result(i)`` returns a dict of the
    outputs, ``status`` and the latency in seconds."""

    def __init__(self, capacity: int, keep_outputs: bool = True, pinned=False):
        """pinned: False (pageable numpy buffers), True (page-locked) or "mixed": request i of a
        decomposition has, by i % 4, all buffers page-locked / a pageable input with page-locked
        outputs / a page-locked input with pageable outputs / page-locked input and sigma with a
        pageable second output; forecast outputs alternate."""
        self.arr = (_Request * max(1, capacity))()
        self.n = 0
        self.keep_outputs = keep_outputs
        self._bufs = []
        self._pool = _PinnedPool() if pinned else None
        self._mixed = pinned == "mixed"

    def _locked(self, role: int) -> bool:
        """role 0: input, 1: first output, 2: second output"""
        if self._pool is None:
            return False
        if not self._mixed:
            return True
        pat = (self.n - 1) % 4
        return {0: True, 1: role != 0, 2: role == 0, 3: role != 2}[pat]

    def _buf(self, shape, src=None, role: int = 0):
        if self._locked(role):
            return self._pool.array(shape, src)
        if src is not None:
            return np.ascontiguousarray(src, dtype=np.float64)
        return np.zeros(shape)

    def _next(self):
        if self.n >= len(self.arr):
            raise IndexError("request block is full")
        r = self.arr[self.n]
        self.n += 1
        return r

    def add_decompose(self, x: np.ndarray, L: int, k: int, series_id: int = 0, seed: int = 0,
                      wcorr: bool = False) -> int:
        r = self._next()
        x = self._buf((len(x),), np.asarray(x, dtype=np.float64))
        N = len(x)
        r.type = REQ_DECOMPOSE_WCORR if wcorr else REQ_DECOMPOSE_RECON
        r.series_id, r.N, r.L, r.k, r.seed = series_id, N, L, k, seed
        r.x = _dp(x)
        bufs = {"x": x}
        if self.keep_outputs:
            ke = max(1, min(k, L, N - L + 1))
            bufs["sigma"] = self._buf((ke,), role=1)
            r.sigma = _dp(bufs["sigma"])
            if wcorr:
                bufs["W"] = self._buf((ke, ke), role=2)
                r.W = _dp(bufs["W"])
            else:
                bufs["groups"] = self._buf((2, N), role=2)
                r.groups = _dp(bufs["groups"])
        self._bufs.append(bufs)
        return self.n - 1

    def _group(self, r, bufs, group):
        if group is not None:
            g = np.ascontiguousarray(group, dtype=np.int32)
            bufs["_group"] = g
            r.group = _ip(g)
            r.n_group = len(g)

    def add_forecast(self, series_id: int, h: int, group: Optional[Sequence[int]] = None) -> int:
        """R-forecast of h steps on a resident series: of the group [0, 1, 2] (resident LRF) or of
        `group` (computed from the resident factors)."""
        r = self._next()
        r.type = REQ_FORECAST
        r.series_id, r.h = series_id, h
        bufs = {}
        self._group(r, bufs, group)
        if self.keep_outputs:
            bufs["forecast"] = self._buf((h,), role=1 + (self.n - 1) % 2)
            r.forecast = _dp(bufs["forecast"])
        self._bufs.append(bufs)
        return self.n - 1

    def add_reconstruct(self, series_id: int, N: int, group: Sequence[int]) -> int:
        """Reconstruction of `group` of a resident series of length N (no decomposition)."""
        r = self._next()
        r.type = REQ_RECONSTRUCT
        r.series_id = series_id
        bufs = {}
        self._group(r, bufs, group)
        if self.keep_outputs:
            bufs["out"] = self._buf((N,), role=1)
            r.out = _dp(bufs["out"])
        self._bufs.append(bufs)
        return self.n - 1

    def add_cadzow(self, rank: int, max_iter: int = 10, tol: float = 1e-9, series_id: int = 0,
                   x: Optional[np.ndarray] = None, L: int = 0, N: Optional[int] = None) -> int:
        """Cadzow iterations of rank `rank`: on the resident series `series_id` (x None; N its length)
        or on the new signal x with window L."""
        r = self._next()
        r.type = REQ_CADZOW
        r.series_id, r.rank, r.max_iter, r.tol = series_id, rank, max_iter, tol
        bufs = {}
        if x is not None:
            xb = self._buf((len(x),), np.asarray(x, dtype=np.float64))
            bufs["x"] = xb
            r.x = _dp(xb)
            r.N, r.L = len(xb), L
            N = len(xb)
        if self.keep_outputs:
            bufs["out"] = self._buf((N,), role=1)
            r.out = _dp(bufs["out"])
        self._bufs.append(bufs)
        return self.n - 1

    def result(self, i: int) -> dict:
        r = self.arr[i]
        out = {k: v for k, v in self._bufs[i].items() if k not in ("x", "_group")}
        if r.type == REQ_CADZOW:
            out["iterations"], out["final_diff"] = r.iterations, r.final_diff
        if "sigma" in out:
            out["sigma"] = out["sigma"][:r.k_out] if r.k_out else out["sigma"][:0]
        out["status"] = r.status
        out["latency"] = r.t_done - r.t_arrival
        return out

    def latencies(self) -> np.ndarray:
        return np.array([self.arr[i].t_done - self.arr[i].t_arrival for i in range(self.n)])

    def statuses(self) -> np.ndarray:
        return np.array([self.arr[i].status for i in range(self.n)])

    def times(self) -> tuple[np.ndarray, np.ndarray]:
        return (np.array([self.arr[i].t_arrival for i in range(self.n)]),
                np.array([self.arr[i].t_done for i in range(self.n)]))


class SSAServer:
    """Continuous-batching request server (ssa_server_* C ABI)."""

    def __init__(self, hbm_budget_bytes: int = 0, max_inflight: int = 3, max_batch: int = 4096,
                 oversampling: int = 10, power_iters: int = 2):
        self._h = ctypes.c_void_p()
        if _lib.ssa_server_create(ctypes.byref(self._h), hbm_budget_bytes, max_inflight, max_batch, oversampling,
                                  power_iters) != 0:
            raise ValueError("ssa_server_create failed")

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.ssa_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        self.close()

    def submit(self, reqs: Requests, i: int) -> None:
        if _lib.ssa_server_submit(self._h, ctypes.byref(reqs.arr[i])) != 0:
            raise RuntimeError("ssa_server_submit failed")

    def drain(self) -> None:
        _lib.ssa_server_drain(self._h)

    def run(self, reqs: Requests, arrivals: Optional[np.ndarray] = None) -> None:
        """Submit every request of the block at its arrival offset (seconds; all at once when
        None) and wait until all have completed."""
        arr = np.zeros(reqs.n) if arrivals is None else np.ascontiguousarray(arrivals, dtype=np.float64)
        if len(arr) != reqs.n:
            raise ValueError("one arrival time per request")
        if _lib.ssa_server_replay(self._h, reqs.arr, _dp(arr), reqs.n) != 0:
            raise RuntimeError("ssa_server_replay failed")

    def stats(self) -> dict:
        st = _ServerStats()
        _lib.ssa_server_stats_get(self._h, ctypes.byref(st))
        return {n: getattr(st, n) for n, _ in _ServerStats._fields_}


def server_now() -> float:
    return float(_lib.ssa_server_now())
