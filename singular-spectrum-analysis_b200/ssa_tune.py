"""Autotuner for the uneven-batch launch parameters (ssa_b200_tune_set).

Per FFT-length bucket it measures the Gram partial launches of a synthetic batch of that
bucket's lengths under candidate CTA counts, with the batch's serialized profiler (every launch's
CUDA-event interval its own), and keeps the fastest; then it chooses the multi-length sweep
setting (one persistent launch for real FFT lengths 512..16384 at one or two CTAs per SM, or one
bucket per length) by the wall time of a mixed batch, and the FFT form of the real length 32768
(one 1024-thread CTA or a cluster of two 8192-point CTAs per transform) by the wall time of a
batch of that bucket. A candidate replaces the built-in heuristic
only when it is faster by more than `margin` (default 3 %), so that run-to-run noise does not flip
choices. The chosen table is written to a JSON cache keyed by the GPU name, its SM count and a
digest of the library; a later call with the same key applies the cached table without measuring.

    import ssa_tune
    table = ssa_tune.autotune()          # measures (about 20-40 s on one B200) or loads the cache
    ssa_tune.apply(table)                # what autotune already did
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import math
import os
import time
from pathlib import Path
from typing import Optional

import numpy as np

import ssa_gpu

_lib = ssa_gpu._lib
_lib.ssa_b200_tune_set.restype = ctypes.c_int
_lib.ssa_b200_tune_set.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int]
_lib.ssa_b200_tune_get.restype = ctypes.c_int
_lib.ssa_b200_tune_get.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
_lib.ssa_b200_fft_size_code.restype = ctypes.c_int
_lib.ssa_b200_fft_size_code.argtypes = [ctypes.c_int]
_lib.ssa_b200_set_cluster32k.restype = None
_lib.ssa_b200_set_cluster32k.argtypes = [ctypes.c_int]
_lib.ssa_b200_cluster32k.restype = ctypes.c_int

NCODES = 20
GRAM_CANDIDATES = (296, 592, 1184, 2368)  # 2, 4, 8 (the heuristic) and 16 CTAs per SM
HEURISTIC_GRAM = 1184
# representative series lengths per tuned bucket (size code): the buckets a mixed stream of N in
# [500, 1e5] uses. With the multi-length sweep on, lengths 513..16384 share the bucket of code 13,
# whose table entry then holds for all of them, so that bucket is tuned on the mixed range.
BUCKET_N = {13: (513, 16384), 14: (16385, 32768), 17: (32769, 49152), 15: (49153, 65536),
            19: (65537, 81920), 18: (81921, 98304), 16: (98305, 131072)}


def size_code(N: int) -> int:
    return int(_lib.ssa_b200_fft_size_code(int(N)))


def current() -> dict:
    g = (ctypes.c_int * NCODES)()
    m = ctypes.c_int()
    _lib.ssa_b200_tune_get(g, NCODES, ctypes.byref(m))
    return {"gram_ctas": list(g), "multi": ssa_gpu.multi_length(), "multi_ctas_per_sm": m.value,
            "cluster32k": bool(_lib.ssa_b200_cluster32k())}


def apply(table: dict) -> None:
    """Set the tuning table (gram_ctas per size code, multi on/off, multi CTAs per SM, the FFT form
    of the real length 32768)."""
    g = (ctypes.c_int * NCODES)(*[int(v) for v in table.get("gram_ctas", [0] * NCODES)][:NCODES])
    if _lib.ssa_b200_tune_set(g, NCODES, int(table.get("multi_ctas_per_sm", 0))) != 0:
        raise ValueError("invalid tuning table")
    ssa_gpu.set_multi_length(bool(table.get("multi", True)))
    _lib.ssa_b200_set_cluster32k(1 if table.get("cluster32k", False) else 0)


def reset() -> None:
    apply({"gram_ctas": [0] * NCODES, "multi": True, "multi_ctas_per_sm": 0, "cluster32k": False})


def cache_key() -> dict:
    """GPU name and SM count (from torch, "unknown" without a GPU) and a digest of libssa.so."""
    props = _device_props()
    lib = Path(ssa_gpu.__file__).resolve().parent / "libssa.so"
    digest = hashlib.sha256(lib.read_bytes()).hexdigest()[:16] if lib.exists() else "unknown"
    return {"gpu": props[0], "sms": props[1], "library": digest}


def _device_props():
    try:
        import torch

        p = torch.cuda.get_device_properties(torch.cuda.current_device())
        return p.name, int(p.multi_processor_count)
    except Exception:
        return "unknown", 0


def default_cache_path() -> Path:
    env = os.environ.get("SSA_TUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "ssa_b200" / "tune.json"


def load(path: Optional[Path] = None) -> Optional[dict]:
    """The cached table for this GPU and library build, or None."""
    path = Path(path) if path else default_cache_path()
    try:
        data = json.loads(path.read_text())
    except (OSError, ValueError):
        return None
    return data if data.get("key") == cache_key() else None


def _series(rng, n: int, lo: int, hi: int):
    xs, Ls, ks = [], [], []
    for _ in range(n):
        N = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        t = np.arange(N)
        x = np.cumsum(rng.standard_normal(N)) * 0.05 + np.sin(2 * np.pi * t / rng.uniform(4, max(5, N / 10)))
        xs.append(x + 0.3 * rng.standard_normal(N))
        Ls.append(max(2, N // 4))
        ks.append(int(rng.integers(10, 51)))
    return xs, Ls, ks


def _gram_ms(rb, xs, Ls, ks, reps: int) -> float:
    """Median over reps of the Gram stage's summed launch time (serialized profiler, ms)."""
    out = []
    rb.set_profiling(True, serialize=True)
    try:
        for r in range(reps + 1):
            rb.profile()
            rb.run(xs, Ls, ks, seed=r)
            prof = rb.profile()
            ms = prof["gram"][0] + prof.get("wcorr_gram", (0.0, 0))[0]
            if r:
                out.append(ms)
    finally:
        rb.set_profiling(False)
    return float(np.median(out))


def _wall_ms(rb, xs, Ls, ks, reps: int) -> float:
    Na = [len(x) for x in xs]
    x = np.concatenate(xs)
    import torch

    d_x = torch.from_numpy(x).to("cuda")
    out = []
    for r in range(reps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rb.run_device(d_x.data_ptr(), Na, Ls, ks, seed=r)
        rb.sync()
        if r:
            out.append((time.perf_counter() - t0) * 1e3)
    return float(np.median(out))


def autotune(cache: Optional[Path] = None, buckets=None, series: int = 96, reps: int = 3, margin: float = 0.03,
             retune: bool = False, seed: int = 0) -> dict:
    """Load the cached table for this GPU and library, or measure one, apply it and cache it.
    buckets: size codes to tune (default: those of BUCKET_N). Returns the table with its
    measurements."""
    cache = Path(cache) if cache else default_cache_path()
    if not retune:
        hit = load(cache)
        if hit is not None:
            apply(hit["table"])
            return hit
    reset()
    rng = np.random.default_rng(seed)
    gram = [0] * NCODES
    meas = {}
    t_start = time.perf_counter()
    # the FFT form of real length 32768: one 1024-thread CTA or a 2-CTA cluster per transform
    cl32 = False
    if buckets is None or 14 in buckets:
        xs, Ls, ks = _series(rng, series, *BUCKET_N[14])
        rb = ssa_gpu.SSARaggedBatch(oversampling=10, power_iters=2)
        forms = {}
        for on in (False, True):
            apply({"gram_ctas": gram, "multi": True, "multi_ctas_per_sm": 0, "cluster32k": on})
            forms[on] = _wall_ms(rb, xs, Ls, ks, reps)
        cl32 = forms[True] < (1.0 - margin) * forms[False]
        meas["cluster32k_wall_ms"] = {"single_cta": round(forms[False], 3), "cluster2": round(forms[True], 3)}
        del rb
    for code in (buckets if buckets is not None else list(BUCKET_N)):
        lo, hi = BUCKET_N[code]
        n = 2 * series if code == 13 else series if code == 14 else max(12, series // 4)
        xs, Ls, ks = _series(rng, n, lo, hi)
        rb = ssa_gpu.SSARaggedBatch(oversampling=10, power_iters=2)
        times = {}
        for cand in GRAM_CANDIDATES:
            g = list(gram)
            g[code] = cand
            apply({"gram_ctas": g, "multi": True, "multi_ctas_per_sm": 0, "cluster32k": cl32})
            times[cand] = _gram_ms(rb, xs, Ls, ks, reps)
        base = times[HEURISTIC_GRAM]
        best = min(times, key=lambda c: (times[c], GRAM_CANDIDATES.index(c)))
        gram[code] = best if times[best] < (1.0 - margin) * base else 0
        meas[str(code)] = {"gram_ms": {str(c): round(t, 4) for c, t in times.items()}, "chosen": gram[code]}
        del rb
    # the multi-length sweep on a mixed batch of the single-CTA lengths
    xs, Ls, ks = _series(rng, 4 * series, 500, 16384)
    rb = ssa_gpu.SSARaggedBatch(oversampling=10, power_iters=2)
    opts = {"off": (False, 0), "on_2": (True, 0), "on_1": (True, 1)}
    wall = {}
    for name, (on, cps) in opts.items():
        apply({"gram_ctas": gram, "multi": on, "multi_ctas_per_sm": cps, "cluster32k": cl32})
        wall[name] = _wall_ms(rb, xs, Ls, ks, reps)
    best = min(wall, key=lambda k: (wall[k], list(opts).index(k)))
    if wall[best] >= (1.0 - margin) * wall["on_2"]:
        best = "on_2"
    table = {"gram_ctas": gram, "multi": opts[best][0], "multi_ctas_per_sm": opts[best][1], "cluster32k": cl32}
    apply(table)
    out = {"key": cache_key(), "table": table, "measurements": {"buckets": meas, "multi_wall_ms": wall},
           "seconds": round(time.perf_counter() - t_start, 1), "margin": margin}
    try:
        cache.parent.mkdir(parents=True, exist_ok=True)
        cache.write_text(json.dumps(out, indent=1))
    except OSError:
        pass
    return out
