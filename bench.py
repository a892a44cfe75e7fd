"""Throughput and latency benchmark of the B200 SSA hot path on the mixed-N serving stream.

Workload (default): requests with N log-uniform in [500, 100000], L = round(N/4), k uniform in
{10..50}, oversampling p = 10, q = 2 power iterations; 50 % decompose + reconstruct groups [0] and
[1, 2] (the series then stays resident), 30 % R-forecast of 50 steps on an already-resident series,
20 % decompose + W-correlation. Signals: seeded random-walk trend + 1-3 sinusoids + Gaussian noise
at SNR U(0, 15) dB (the uneven-batch generator). One SSA = one served request.

Output: one JSON line (rank 0).
  value  series/s of the uneven-batch pipeline over the stream's decompositions with inputs
         resident in HBM (CUDA events on the batch's stream; inputs larger than L2);
  e2e    requests/s of the request server (ssa_server_*, host buffers, H2D and D2H inside) with the
         whole stream offered at once;
  latency_ms  p50 / p99 arrival-to-result latency at Poisson arrival rates 1k-50k requests/s;
  plain_gpu_path  the same stream one request per call through the reference-compatible API;
  cpu_baseline    the reference's CPU implementation on a bounded sample of the stream.
`--impl reference` times the reference's CPU implementation instead.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

if mp.current_process().name != "MainProcess":
    # pool workers (CPU baseline, accuracy checks): one BLAS thread each, set before numpy loads it
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"

import numpy as np

# one hardware work queue per stream for the bucket streams of the batches in flight (the
# runtime's default of 8 serialises streams that share a queue); read when the CUDA context is
# created, so it is set before anything touches the GPU
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "singular-spectrum-analysis_b200"
ORACLE = ROOT / "oracle"
for _p in (str(PKG), str(ORACLE)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--batch", type=int, default=2048, help="series per device step")
    ap.add_argument("--requests", type=int, default=4096, help="stream length for the saturated server run")
    ap.add_argument("--rates", default="1000,2000,5000,10000,20000,50000")
    ap.add_argument("--nmin", type=int, default=500)
    ap.add_argument("--nmax", type=int, default=100000)
    ap.add_argument("--p", type=int, default=10)
    ap.add_argument("--q", type=int, default=2)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-uniform", action="store_true")
    ap.add_argument("--no-config4", action="store_true")
    ap.add_argument("--no-rates", action="store_true")
    ap.add_argument("--accuracy", type=int, default=64, help="series of the timed batch checked against the FP64 "
                                                              "oracle after the run (0: none)")
    return ap.parse_args()


def workload_config(a) -> dict:
    return {"workload": f"mixed-N serving stream: N log-uniform [{a.nmin}, {a.nmax}], L = N/4, k ~ U{{10..50}}, "
                        f"p = {a.p}, q = {a.q}; 50% decompose + reconstruct [0],[1,2] (series stays resident), "
                        "30% R-forecast 50 steps on a resident series, 20% decompose + W-correlation",
            "series_per_step": a.batch, "stream_requests": a.requests, "oversampling": a.p, "power_iters": a.q,
            "rates_per_s": [int(r) for r in a.rates.split(",")], "seed": a.seed,
            "l2": "inputs larger than L2 (packed signals of a step: ~300 MB)",
            "parallelism": "series sharded per GPU, no collective"}


# ------------------------------------------------------------------------------------------
# the stream
# ------------------------------------------------------------------------------------------

RECON, WCORR, FORECAST = 0, 1, 2


def make_series(rng: np.random.Generator, nmin: int, nmax: int):
    import ssa_oracle

    N = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
    L = max(2, int(round(N / 4)))
    k = int(rng.integers(10, 51))
    return ssa_oracle.walk_sines(rng, N), L, k


def make_stream(n: int, seed: int, nmin: int, nmax: int) -> list:
    """Request specs: (type, x, L, k, target) in arrival order; a forecast names the index of an
    earlier decompose + reconstruct request."""
    rng = np.random.default_rng(seed)
    out, recon_idx = [], []
    for i in range(n):
        u = rng.random()
        t = RECON if u < 0.5 else (FORECAST if u < 0.8 else WCORR)
        if t == FORECAST and not recon_idx:
            t = RECON
        if t == FORECAST:
            out.append((FORECAST, None, 0, 0, recon_idx[int(rng.integers(0, len(recon_idx)))]))
        else:
            x, L, k = make_series(rng, nmin, nmax)
            out.append((t, x, L, k, -1))
            if t == RECON:
                recon_idx.append(i)
    return out


def stream_requests(gpu, specs, id_base: int, keep_outputs: bool = True, pinned: bool = True):
    """Request block for the server; inputs and outputs in page-locked host memory. Returns the
    block and the bytes it moves host -> device and device -> host."""
    R = gpu.Requests(len(specs), keep_outputs=keep_outputs, pinned=pinned)
    h2d = d2h = 0
    for i, (t, x, L, k, tgt) in enumerate(specs):
        if t == FORECAST:
            R.add_forecast(id_base + tgt, 50)
            d2h += 8 * 50 if keep_outputs else 0
        else:
            R.add_decompose(x, L, k, series_id=id_base + i, seed=id_base + i, wcorr=(t == WCORR))
            N = len(x)
            ke = min(k, L, N - L + 1)
            h2d += 8 * N
            if keep_outputs:
                d2h += 8 * (ke + (ke * ke if t == WCORR else 2 * N))
    return R, h2d, d2h


# DRAM traffic of the correlation sweeps measured by ncu relative to their algorithmic bytes:
# k_corr<13> 0.985 (uniform 512-series batch), k_cl_col<6, CL_CORR> 1.002 and 0.980 (mixed
# 512-series batch, real FFT length 98304); the mean is used to state the traffic of a launch.
CORR_TRAFFIC_RATIO = 0.989
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # SMs x FP32 lanes x FMA x clock (nominal peak)


def corr_flops(N: int, L: int, k: int, p: int, q: int, M: int) -> float:
    """Algorithmic FLOPs of the correlation sweeps of one series at real FFT length M: per probe
    column a forward and an inverse complex FFT of H = M/2 points (5 H log2 H each, the usual
    count for any length) and the real-spectrum unpacking, spectral product and packing (~12 H)."""
    K = N - L + 1
    kp = min(k + p, L, K)
    H = M // 2
    return (2 * q + 2) * kp * (10.0 * H * math.log2(H) + 12.0 * H)


def elem_bytes(N: int, L: int, k: int, p: int, want_w: bool) -> int:
    """Algorithmic FP32 bytes of the elementary reconstructions of one series: per computed
    component its sigma u (L) and v (K) columns read and its N-point reconstruction written (all k
    components for a W-correlation request, components 0..2 for groups [0], [1, 2])."""
    K = N - L + 1
    kk = min(k, k + p, L, K)
    n = kk if want_w else min(kk, 3)
    return 4 * n * (L + K + N)


def corr_bytes(N: int, L: int, k: int, p: int, q: int) -> int:
    """Algorithmic FP32 bytes of the correlation sweeps of one series: the generated first sweep
    writes Y (L x kp); every other sweep reads one block and writes the other."""
    K = N - L + 1
    kp = min(k + p, L, K)
    return 4 * kp * (L + (2 * q + 1) * (L + K))


# ------------------------------------------------------------------------------------------
# CPU reference leg (rank 0 only): the reference's own MKL/ssa_opt.h, compiled unmodified against
# the MKL-compatibility shim (oracle/_ref/libssa_mklshim.so: CBLAS/LAPACKE from OpenBLAS, own
# FFT for DFTI), when present; else the NumPy FP64 port of the same algorithm.
# ------------------------------------------------------------------------------------------

_MKR = None


def _mkr():
    global _MKR
    if _MKR is None:
        import ctypes
        lib = ctypes.CDLL(str(ORACLE / "_ref" / "libssa_mklshim.so"))
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        c_int = ctypes.c_int
        lib.mkr_pipeline.argtypes = [dp, c_int, c_int, c_int, c_int, ip, ip, c_int, dp, c_int, dp, ip, c_int,
                                     c_int, dp, dp, dp, dp]
        lib.mkr_forecast_resident.argtypes = [dp, c_int, c_int, c_int, c_int, ip, c_int, c_int, dp, dp]
        _MKR = (lib, dp, ip)
    return _MKR


def _ref_worker(args):
    """One stream request through the reference's call sequence (the Python wrapper's: init ->
    prepare(k, p) -> decompose_randomized(k, p) -> reconstruct [0], [1, 2] | wcorr_matrix; a
    forecast request: ssa_opt_forecast([0, 1, 2], 50) on an already decomposed context, timed
    alone). Returns the request's seconds."""
    import ctypes
    t, x, L, k, p = args
    lib, dp, ip = _mkr()
    N = len(x)
    x = np.ascontiguousarray(x, dtype=np.float64)
    D = lambda a: a.ctypes.data_as(dp)  # noqa: E731
    I = lambda a: a.ctypes.data_as(ip)  # noqa: E731
    g3 = np.array([0, 1, 2], dtype=np.int32)
    if t == FORECAST:
        fc = np.zeros(50)
        sec = ctypes.c_double(0.0)
        lib.mkr_forecast_resident(D(x), N, L, k, p, I(g3), 3, 50, D(fc), ctypes.byref(sec))
        return sec.value
    sizes = np.array([1, 2], dtype=np.int32)
    sig = np.zeros(k)
    t0 = time.perf_counter()
    if t == RECON:
        rec = np.zeros(2 * N)
        lib.mkr_pipeline(D(x), N, L, k, p, I(g3), I(sizes), 2, D(rec), 0, None, None, 0, 0, None, None, None, D(sig))
    else:
        W = np.zeros(k * k)
        lib.mkr_pipeline(D(x), N, L, k, p, None, None, 0, None, 1, D(W), None, 0, 0, None, None, None, D(sig))
    return time.perf_counter() - t0


def _port_worker(args):
    t, x, L, k, p = args
    import ssa_oracle as O
    N = len(x)
    rng = np.random.default_rng(0)
    Om = O.gaussian_omega(rng, N - L + 1, min(k + p, L, N - L + 1))
    d = O.decompose_randomized(x, L, k, p, Om, q=0)
    t0 = time.perf_counter()
    if t == FORECAST:
        O.forecast(d, [0, 1, 2], 50, N, L)
        return time.perf_counter() - t0
    if t == RECON:
        O.reconstruct(d, [0], N, L)
        O.reconstruct(d, [1, 2], N, L)
    else:
        O.wcorr_matrix(d, N, L)
    return time.perf_counter() - t0


def _spread_order(n: int) -> list:
    """0..n-1 in bit-reversed (van der Corput) order: every prefix is spread evenly over the
    range, so a time-bounded prefix of requests sorted by N samples the stream's N quantiles."""
    bits = max(1, (n - 1).bit_length())
    out = []
    for i in range(1 << bits):
        r = int(format(i, f"0{bits}b")[::-1], 2)
        if r < n:
            out.append(r)
    return out


def cpu_reference(a, budget_s: float = 20.0) -> dict:
    """Time the reference CPU path on a bounded sample of the stream's requests: one request per
    process on every host core (each process single-threaded, OpenBLAS included), requests taken
    in an order that spreads over the stream's sorted N, as many as fit the budget. Forecast
    requests are timed as the forecast call on a resident (already decomposed) series.
    Returns {"value", "unit", "cores", "kind", "sample"}."""
    cores = len(os.sched_getaffinity(0))
    use_ref = (ORACLE / "_ref" / "libssa_mklshim.so").exists()
    specs = make_stream(a.requests, a.seed, a.nmin, a.nmax)
    reqs = []
    for t, x, L, k, tgt in specs:
        if t == FORECAST:
            _, x, L, k, _ = specs[tgt]
        reqs.append((t, x, L, k))
    order = sorted(range(len(reqs)), key=lambda i: len(reqs[i][1]))
    pick = [order[i] for i in _spread_order(len(order))]
    ctx = mp.get_context("spawn")
    done, busy, nsum = 0, 0.0, 0
    worker = _ref_worker if use_ref else _port_worker
    with ctx.Pool(cores, initializer=_pin_blas) as pool:
        pool.map(_pin_blas, range(cores))  # workers started before the clock
        t0 = time.perf_counter()
        pos = 0
        while pos < len(pick):
            batch = [reqs[i] for i in pick[pos:pos + cores]]
            pos += len(batch)
            secs = pool.map(worker, [(t, x, L, k, a.p) for t, x, L, k in batch])
            busy += sum(secs)
            done += len(batch)
            nsum += sum(len(b[1]) for b in batch)
            if time.perf_counter() - t0 >= budget_s:
                break
        wall = time.perf_counter() - t0
    # requests/s with every core busy: cores / mean seconds per request (the wall-clock rate of the
    # batches, which wait for their slowest request, is reported beside it)
    value = cores * done / busy if busy > 0 else 0.0
    kind = "reference" if use_ref else "port"
    what = ("the reference's MKL/ssa_opt.h compiled unmodified against an MKL-compatibility shim (OpenBLAS "
            "CBLAS/LAPACKE, own power-of-two real FFT for DFTI; no MKL on this host): randomized SVD with the "
            "reference's q = 0, uncached reconstructions [0],[1,2], ssa_opt_wcorr_matrix, ssa_opt_forecast"
            if use_ref else "NumPy FP64 port of MKL/ssa_opt.h randomized SVD (q = 0), reconstruct, W-corr, forecast")
    mean_stream = float(np.mean([len(r[1]) for r in reqs]))
    return {"value": value, "unit": "SSA/s", "cores": cores, "kind": kind,
            "sample": f"{done} of the stream's {len(reqs)} requests (mean N {nsum / max(done, 1):.0f}, stream mean "
                      f"{mean_stream:.0f}; taken spread over the stream's N quantiles) in {busy:.1f} core-seconds, one "
                      f"single-threaded process per core on {cores} cores (wall-clock rate of the batches "
                      f"{done / wall:.1f}/s); {what}"}


def _pin_blas(*_):
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"


# ------------------------------------------------------------------------------------------
# accuracy of the timed outputs against the FP64 oracle (CPU, spawn pool; after the timed region)
# ------------------------------------------------------------------------------------------

DENSE_MAX_N = 6000  # exact dense SVD of the trajectory matrix below this length (seconds each)


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _accuracy_worker(args):
    """Errors of one series' GPU outputs against the FP64 restatement of the same algorithm with
    the same device-generated test matrix (and against the exact dense SVD for short series)."""
    import ssa_oracle as O
    from scipy.linalg import subspace_angles
    x, L, k, p, q, seed_s, g = args
    N = len(x)
    K = N - L + 1
    kk, kp = O.clamp_kp(L, K, k, p)
    d = O.decompose_randomized(x, L, kk, p, O.device_gaussian(seed_s, K, kp), q=q)
    sg = g["sigma"]
    rel = np.abs(sg - d.sigma) / d.sigma
    lead = min(3, kk)
    out = {"N": N, "k": kk, "sigma_rel_max": float(rel.max()), "sigma_rel_lead": float(rel[:lead].max()),
           "angle_lead": float(np.max(subspace_angles(g["U"][:, :lead], d.U[:, :lead]))),
           "angle_k": float(np.max(subspace_angles(g["U"], d.U)))}
    recs = []
    for gi, grp in enumerate(([0], [1, 2])):
        if max(grp) < kk:
            recs.append(_rel_l2(g["groups"][gi], O.reconstruct(d, grp, N, L)))
    out["recon_rel"] = max(recs) if recs else 0.0
    if g.get("W") is not None:
        out["W_abs"] = float(np.max(np.abs(g["W"] - O.wcorr_matrix(d, N, L))))
    if N <= DENSE_MAX_N:
        t = O.dense_svd(x, L, kk)
        out["dense_sigma_rel_lead"] = float(np.max(np.abs(sg[:lead] - t.sigma[:lead]) / t.sigma[:lead]))
        out["dense_angle_lead"] = float(np.max(subspace_angles(g["U"][:, :lead], t.U[:, :lead])))
        if lead == 3:
            out["dense_recon_rel"] = max(_rel_l2(g["groups"][0], O.reconstruct(t, [0], N, L)),
                                         _rel_l2(g["groups"][1], O.reconstruct(t, [1, 2], N, L)))
    return out


def _forecast_worker(args):
    import ssa_oracle as O
    x, L, k, p, q, seed_s, fc = args
    N = len(x)
    K = N - L + 1
    kk, kp = O.clamp_kp(L, K, k, p)
    d = O.decompose_randomized(x, L, kk, p, O.device_gaussian(seed_s, K, kp), q=q)
    ref = O.forecast(d, [0, 1, 2], len(fc), N, L)
    return {"rmse": float(np.sqrt(np.mean((fc - ref) ** 2))),
            "rel": float(np.sqrt(np.mean((fc - ref) ** 2)) / max(np.sqrt(np.mean(ref ** 2)), 1e-300))}


def stratified_sample(Ns, n: int, fft_length) -> list:
    """n series indices spread over the FFT-length buckets: every bucket contributes in
    proportion to its series count, at least two where it has them."""
    by = {}
    for i, N in enumerate(Ns):
        by.setdefault(fft_length(N), []).append(i)
    keys = sorted(by)
    take = {b: min(len(by[b]), max(2, round(n * len(by[b]) / len(Ns)))) for b in keys}
    out = []
    for b in keys:
        idx = by[b]
        step = len(idx) / take[b]
        out += [idx[int(j * step)] for j in range(take[b])]
    return sorted(out)


def summarize_accuracy(rows: list, fcs: list) -> dict:
    def agg(key):
        v = np.array([r[key] for r in rows if key in r])
        return {"max": float(v.max()), "p99": float(np.percentile(v, 99)), "n": int(v.size)} if v.size else None
    out = {"series": len(rows), "what": "GPU outputs of the timed batch (and of the server run for forecasts) against "
                                         "the FP64 restatement of the same algorithm with the same device test matrix "
                                         "(q as timed); dense_* against the exact dense SVD of the trajectory matrix "
                                         f"for N <= {DENSE_MAX_N}; angles in radians"}
    for key in ("sigma_rel_lead", "sigma_rel_max", "recon_rel", "W_abs", "angle_lead", "angle_k",
                "dense_sigma_rel_lead", "dense_angle_lead", "dense_recon_rel"):
        a = agg(key)
        if a:
            out[key] = a
    if fcs:
        out["forecast_rmse_rel"] = {"max": max(f["rel"] for f in fcs), "p99": float(np.percentile([f["rel"] for f in fcs], 99)),
                                    "n": len(fcs), "what": "RMSE of 50-step R-forecasts of group [0,1,2] / RMS of the oracle's"}
        out["forecast_rmse"] = {"max": max(f["rmse"] for f in fcs)}
    return out


# ------------------------------------------------------------------------------------------
# clocks sampling during the timed region
# ------------------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([c.strip() for c in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for n, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def measured_peak_hbm() -> tuple[float, str]:
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ------------------------------------------------------------------------------------------
# main
# ------------------------------------------------------------------------------------------

def device_steps(gpu, torch, a, rank: int, world: int) -> dict:
    """Uneven-batch pipeline over `a.batch` stream decompositions with inputs resident in HBM."""
    rng = np.random.default_rng(a.seed + 7919 * (rank + 1))
    series = [make_series(rng, a.nmin, a.nmax) for _ in range(a.batch)]
    # request type of each decomposition as in the stream (50 % reconstruct : 20 % W-correlation):
    # W-correlation requests get W (all elementary reconstructions), reconstruct requests their
    # groups [0], [1, 2]
    want_w = rng.random(a.batch) < 2.0 / 7.0
    Ns = [len(x) for x, _, _ in series]
    Ls = [L for _, L, _ in series]
    ks = [k for _, _, k in series]
    d_x = torch.from_numpy(np.concatenate([x for x, _, _ in series])).to("cuda")
    rb = gpu.SSARaggedBatch(oversampling=a.p, power_iters=a.q, groups=[[0], [1, 2]])
    stream = torch.cuda.ExternalStream(rb.device_results()["stream"])
    for w in range(a.warmup):
        rb.run_device(d_x.data_ptr(), Ns, Ls, ks, seed=1000 + w, want_w=want_w)
        rb.sync()
    launches0 = gpu.kernel_launches()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    with ClockSampler(torch.cuda.current_device()) as clk:
        ev[0].record(stream)
        for i in range(a.steps):
            rb.run_device(d_x.data_ptr(), Ns, Ls, ks, seed=i, want_w=want_w)
            ev[i + 1].record(stream)
        torch.cuda.synchronize()
        rb.sync()
    launches = gpu.kernel_launches() - launches0
    step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(a.steps)]
    total_ms = ev[0].elapsed_time(ev[a.steps])
    # outputs of the last timed step for a stratified sample (checked on the CPU at the end)
    acc_jobs = []
    if rank == 0 and a.accuracy > 0:
        import ssa_oracle
        last_seed = a.steps - 1
        for i in stratified_sample(Ns, a.accuracy, gpu.fft_length):
            r = rb.series_result(i, Ns[i], Ls[i], ks[i], factors=True)
            g = {"sigma": r["sigma"], "groups": r["groups"], "U": r["U"], "W": r["W"] if want_w[i] else None}
            acc_jobs.append((series[i][0], Ls[i], ks[i], a.p, a.q, ssa_oracle.series_seed(last_seed, i), g))
    # one more (untimed) step with the buckets run one after another and every launch bracketed by
    # CUDA events on its stream: isolated per-launch times for the roofline and the kernel shares
    rb.set_profiling(True, serialize=True)
    rb.profile()
    rb.run_device(d_x.data_ptr(), Ns, Ls, ks, seed=999, want_w=want_w)
    rb.sync()
    prof = rb.profile()
    rb.set_profiling(False)
    if world > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    cb = sum(corr_bytes(N, L, k, a.p, a.q) for N, L, k in zip(Ns, Ls, ks))
    cf = sum(corr_flops(N, L, k, a.p, a.q, gpu.fft_length(N)) for N, L, k in zip(Ns, Ls, ks))
    # the same flops at the shortest transform a linear correlation of N points needs (M = N,
    # rounded to even): padding to the FFT lengths the kernels use does not count as work
    cf_min = sum(corr_flops(N, L, k, a.p, a.q, N + (N & 1)) for N, L, k in zip(Ns, Ls, ks))
    eb = sum(elem_bytes(N, L, k, a.p, bool(w)) for N, L, k, w in zip(Ns, Ls, ks, want_w))
    elem_ms, elem_n = prof.get("elem_recon", (0.0, 0))
    corr_ms, corr_n = prof["corr"]
    peak, peak_kind = measured_peak_hbm()
    per_launch = cb / max(corr_n, 1)
    avg_ms = corr_ms / max(corr_n, 1)
    achieved = per_launch / (avg_ms / 1e3) / 1e9
    tflops = cf / (corr_ms / 1e3) / 1e12 if corr_ms > 0 else 0.0
    tflops_min = cf_min / (corr_ms / 1e3) / 1e12 if corr_ms > 0 else 0.0
    elem_gbs = eb / (elem_ms / 1e3) / 1e9 if elem_ms > 0 else 0.0
    tot = max(sum(v[0] for v in prof.values()), 1e-9)
    out = {"value": a.batch * a.steps * world / (total_ms / 1e3), "ms_per_step": total_ms / a.steps,
           "step_ms": step_ms, "launches": launches, "acc_jobs": acc_jobs,
           "share": {kk: round(v[0] / tot, 4) for kk, v in prof.items() if v[1]},
           "share_what": "per-kernel-kind share of one step with the buckets run one after another",
           "mean_N": float(np.mean(Ns)), "clocks": clk.summary(),
           "roofline": {"bound": "hbm", "kernel": "k_corr / k_cl_col<CL_CORR> (FFT correlation matvec sweeps)",
                        "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_source": peak_kind, "traffic": CORR_TRAFFIC_RATIO * per_launch,
                        "traffic_source": "ncu dram__bytes_read+write / algorithmic bytes of captured launches "
                                          "(k_corr<13> 0.985, k_cl_col<6,1> 1.002 / 0.980) x this launch's bytes",
                        "avg_launch_ms": avg_ms, "algorithmic_bytes_per_launch": per_launch,
                        "compute": {"bound": "fp32 issue", "achieved_tflops": tflops_min,
                                    "achieved_tflops_at_used_lengths": tflops,
                                    "peak_tflops": FP32_NOMINAL_TFLOPS,
                                    "peak_source": "nominal FP32 SIMT peak (148 SMs x 128 lanes x 2 x 1.965 GHz)",
                                    "frac": tflops_min / FP32_NOMINAL_TFLOPS,
                                    "what": "FFT flops (10 H log2 H + 12 H per probe column and sweep) counted at "
                                            "H = N/2, the shortest linear-correlation length, over the correlation "
                                            "launches' CUDA-event time; at the padded lengths the kernels use: "
                                            "achieved_tflops_at_used_lengths"},
                        "note": "per-launch CUDA-event times of one extra step with the FFT-length buckets "
                                "run one after another (the timed steps overlap them)"},
           "roofline_elem_recon": {"bound": "hbm", "kernel": "k_elem_recon / k_elem_recon1 / k_cl_col<C,CL_ELEM>",
                                   "achieved": elem_gbs, "peak": peak, "unit": "GB/s", "frac": elem_gbs / peak,
                                   "peak_source": peak_kind, "launches": elem_n, "ms": elem_ms,
                                   "what": "4 n (L + K + N) bytes per series (n computed components: k for W, else 3) "
                                           "over the elementary-reconstruction launches' CUDA-event time"}}
    del rb, d_x
    torch.cuda.empty_cache()
    return out


def server_runs(gpu, torch, a, rank: int, world: int) -> dict:
    """Saturated server run over the whole stream (e2e) and the latency sweep (rank 0)."""
    specs = make_stream(a.requests, a.seed + 31 * rank, a.nmin, a.nmax)
    srv = gpu.SSAServer(hbm_budget_bytes=150 * 10**9, max_inflight=3, max_batch=4096, oversampling=a.p,
                        power_iters=a.q)
    # warm-up: the whole stream once (every batch slot grows its device buffers to full size)
    W, _, _ = stream_requests(gpu, specs, id_base=10**7)
    for _ in range(2):
        srv.run(W)
    R, h2d, d2h = stream_requests(gpu, specs, id_base=2 * 10**7)
    st0 = srv.stats()
    srv.run(R)
    st1 = srv.stats()
    timed = {kk: st1[kk] - st0[kk] for kk in ("batches", "decompositions", "forecast_batches", "forecasts",
                                                "host_launch_s", "host_finish_s")}
    ta, td = R.times()
    st = R.statuses()
    el = float(td.max() - ta.min())
    fc_jobs = []
    if rank == 0 and a.accuracy > 0:
        fidx = [i for i, sp in enumerate(specs) if sp[0] == FORECAST and st[i] == 0]
        for i in fidx[:: max(1, len(fidx) // 32)][:32]:
            tgt = specs[i][4]
            _, x, L, k, _ = specs[tgt]
            fc_jobs.append((x, L, k, a.p, a.q, 2 * 10**7 + tgt, np.array(R.result(i)["forecast"])))
    if world > 1:
        t = torch.tensor([el], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        el = float(t.item())
    out = {"e2e": {"value": len(specs) * world / el, "unit": "SSA/s", "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h, "requests": len(specs), "failed": int((st != 0).sum()),
                   "seconds": el, "server_timed_run": timed,
                   "what": "ssa_server_* C API, page-locked host buffers, the whole stream offered at t=0 (one "
                           "step = the stream): H2D of every signal and D2H of every requested result (sigma, "
                           "groups [0],[1,2] / W, forecasts) inside the timed region"}, "fc_jobs": fc_jobs}
    if rank == 0 and world == 1 and not a.no_rates:
        sweep = {}
        rng = np.random.default_rng(a.seed + 99)
        for ri, rate in enumerate(int(r) for r in a.rates.split(",")):
            n = min(len(specs), max(400, int(rate * 0.8)))
            Rr, _, _ = stream_requests(gpu, specs[:n], id_base=(3 + ri) * 10**7)
            arr = np.cumsum(rng.exponential(1.0 / rate, n))
            srv.run(Rr, arr)
            ta, td = Rr.times()
            lat = (td - ta) * 1e3
            ok = Rr.statuses() == 0
            sweep[str(rate)] = {"requests": n, "achieved_per_s": n / float(td.max() - ta.min()),
                                "p50_ms": float(np.percentile(lat[ok], 50)), "p99_ms": float(np.percentile(lat[ok], 99)),
                                "failed": int((~ok).sum())}
        sustained = [r for r, v in sweep.items() if v["achieved_per_s"] >= 0.9 * int(r)]
        best = max(sustained, key=int) if sustained else min(sweep, key=int)
        out["latency_ms"] = {"p50": sweep[best]["p50_ms"], "p99": sweep[best]["p99_ms"], "at_rate_per_s": int(best),
                             "what": "arrival-to-result latency (host clock) at the highest swept Poisson rate the "
                                     "server sustains (achieved >= 90% of offered)", "sweep": sweep}
    srv.close()
    return out


def plain_path(gpu, a, n: int = 120, recycle: bool = True) -> dict:
    """The stream's first n requests one per call through the reference-compatible API, a context
    created and freed per decomposition as the reference's wrapper does; with `recycle` the
    library's context recycling (streams, pooled buffers, page-locked staging of freed contexts)
    is on, as by default, else every context allocates afresh."""
    gpu.set_context_recycling(recycle)
    specs = make_stream(n, a.seed, a.nmin, a.nmax)
    objs, lat, failed = {}, [], 0
    t0 = time.perf_counter()
    for i, (t, x, L, k, tgt) in enumerate(specs):
        ts = time.perf_counter()
        try:
            if t == FORECAST:
                objs[tgt].forecast([0, 1, 2], 50)
            else:
                s = gpu.SSA(x, L)
                s.decompose(k, oversampling=a.p, power_iters=a.q)
                if t == RECON:
                    s.reconstruct([0])
                    s.reconstruct([1, 2])
                    objs[i] = s
                else:
                    s.wcorr_matrix()
        except (RuntimeError, KeyError):
            failed += 1
        lat.append((time.perf_counter() - ts) * 1e3)
    el = time.perf_counter() - t0
    objs.clear()
    gpu.set_context_recycling(True)
    return {"value": n / el, "unit": "SSA/s", "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "failed": failed, "context_recycling": recycle,
            "what": f"first {n} requests of the stream, one per call (SSA() + decompose(q={a.q}) + reconstruct x2 "
                    "/ wcorr_matrix / forecast on the kept context) through libssa.so's reference API, host wall "
                    "clock; " + ("contexts recycled (default)" if recycle else "every context allocated afresh")}


def uniform_batch(gpu, torch, a, B: int = 4096, N: int = 10000, L: int = 2500, k: int = 50, steps: int = 3) -> dict:
    """The uniform batch of identical series (4096 x N=10000), for comparison with earlier lines."""
    import ssa_oracle

    X = ssa_oracle.config2_batch(B, seed=1, N=N)
    d_x = torch.from_numpy(X).to("cuda")
    batch = gpu.SSABatch(B, N, L, k, oversampling=a.p, power_iters=a.q, groups=[[0], [1, 2]])
    stream = torch.cuda.ExternalStream(batch.device_results()["stream"])
    for w in range(3):
        batch.run_device(d_x.data_ptr(), B, seed=1000 + w)
        batch.sync()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(steps):
        batch.run_device(d_x.data_ptr(), B, seed=i)
    e1.record(stream)
    torch.cuda.synchronize()
    batch.sync()
    ms = e0.elapsed_time(e1)
    del batch, d_x
    torch.cuda.empty_cache()
    return {"value": B * steps / (ms / 1e3), "unit": "SSA/s", "ms_per_step": ms / steps,
            "workload": f"{B} series x N={N}, L={L}, k={k}, p={a.p}, q={a.q}; decompose + all elementary "
                        "reconstructions + W-correlation + groups [0],[1,2]; inputs resident in HBM"}


def wgram_variants(gpu, a, B: int = 512, N: int = 10000, L: int = 2500, k: int = 50) -> dict:
    """The W-correlation Gram in each of its arithmetics (FP64, split TF32 and split BF16 on the
    tensor cores, FP32 on the CUDA cores) on the uniform batch (B series x N, k components): the
    Gram stage's CUDA-event time, its algorithmic rate (k N floats read per series; k (k + 1) N
    flops per series for the packed upper triangle) and the largest |W - W_fp64|."""
    import ssa_oracle

    X = ssa_oracle.config2_batch(B, seed=21, N=N)
    out, ref = {}, None
    try:
        for mode in (gpu.WGRAM_FP64, gpu.WGRAM_TF32X3, gpu.WGRAM_BF16X3, gpu.WGRAM_FP32):
            gpu.set_wcorr_gram(mode)
            b = gpu.SSABatch(B, N, L, k, oversampling=a.p, power_iters=a.q, groups=[[0]])
            b.run(X, seed=3)  # warm-up
            b.set_profiling(True)
            b.profile()
            _, W, _ = b.run(X, seed=3)
            ms, n = b.profile()["wcorr_gram"]
            b.set_profiling(False)
            del b
            if ref is None:
                ref = W
            kk = W.shape[1]
            byts, flops = 4.0 * kk * N * B, float(kk) * (kk + 1) * N * B
            out[gpu.WGRAM_NAMES[mode]] = {"ms": ms, "launches": n, "GB_s": byts / (ms / 1e3) / 1e9,
                                          "TFLOP_s": flops / (ms / 1e3) / 1e12,
                                          "max_abs_dW_vs_fp64": float(np.max(np.abs(W - ref)))}
    finally:
        gpu.set_wcorr_gram(gpu.WGRAM_TF32X3)
    out["workload"] = (f"W-correlation Gram of {B} series x N={N} (L={L}, k={k}): elementary reconstructions "
                       f"{4 * k * N * B / 1e9:.2f} GB read per launch (> L2); CUDA events on the batch stream")
    return out


def config4(gpu, torch, a, I: int = 64, M: int = 16, N: int = 20000, L: int = 5000, k: int = 50,
            iters: int = 10) -> dict:
    """The multichannel workload: I instances of M correlated channels (random mixings of 4 shared
    sinusoids + trend + noise at SNR 5 dB), block power of each stacked (M L) x K operator (one
    block of kp columns, q subspace iterations) and `iters` multivariate Cadzow iterations of rank
    k, all instances in one batch; inputs resident in HBM."""
    import ssa_oracle

    rng = np.random.default_rng(3)
    X = np.stack([ssa_oracle.config4_instance(rng, Mch=M, N=N) for _ in range(I)])
    d_x = torch.from_numpy(X).to("cuda")
    d_out = torch.empty_like(d_x)
    mb = gpu.SSAMultiBatch(I, M, N, L, k, oversampling=a.p, power_iters=a.q)
    stream = torch.cuda.ExternalStream(mb.stream)
    # warm-up with the timed iteration count (a first run of `iters` iterations carries one-time
    # set-up the one-iteration run does not: ~1.2 s against ~0.72 s measured)
    mb.run_device(d_x.data_ptr(), iters, seed=7, d_out_ptr=d_out.data_ptr())
    mb.sync()
    torch.cuda.synchronize()
    # three timed runs of the whole batch (the same inputs each time); the median is reported
    runs_ms, launches = [], 0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = gpu.kernel_launches()
        e0.record(stream)
        mb.run_device(d_x.data_ptr(), iters, seed=7, d_out_ptr=d_out.data_ptr())
        e1.record(stream)
        mb.sync()
        runs_ms.append(e0.elapsed_time(e1))
        launches = gpu.kernel_launches() - launches0
    ms = float(np.median(runs_ms))
    diff = mb.diffs(iters)
    K = N - L + 1
    kp, kk = mb.kp, mb.k
    # algorithmic FP32 bytes of one Cadzow iteration of one instance: the block sweeps
    # ((2 q + 3) kp columns of the K + M L rows), the factors written and read, the M channels in
    # and out
    per_iter = 4 * ((2 * a.q + 3) * kp * (K + M * L) + 2 * kk * (K + M * L) + 2 * M * N)
    total = per_iter * I * iters
    peak, peak_kind = measured_peak_hbm()
    achieved = total / (ms / 1e3) / 1e9
    out = {"value": I / (ms / 1e3), "unit": "instances/s", "ms_per_instance": ms / I, "ms": ms,
           "ms_per_cadzow_iteration": ms / iters, "launches": launches, "runs_ms": runs_ms,
           "final_rel_change": {"median": float(np.median(diff[:, -1])), "max": float(diff[:, -1].max())},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_source": peak_kind, "algorithmic_bytes": total,
                        "what": "4 [(2q+3) kp (K + M L) + 2 k (K + M L) + 2 M N] bytes per instance per Cadzow "
                                "iteration / whole-run CUDA-event time (median of three runs)"},
           "workload": f"{I} instances x {M} channels, N={N}, L={L}, rank {kk}, block of kp={kp} columns, q={a.q} "
                       f"subspace iterations per projection, {iters} Cadzow iterations; inputs resident in HBM"}
    del mb, d_x, d_out
    torch.cuda.empty_cache()
    return out


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    metric = "SSA/sec (mixed-N serving stream)"
    cfg = workload_config(a)

    if a.impl == "reference":
        if rank != 0:
            return
        steps = []
        for i in range(a.warmup + a.steps):
            r = cpu_reference(a, budget_s=8.0)
            if i >= a.warmup:
                steps.append(r)
        v = statistics.median([s["value"] for s in steps])
        line = {"impl": "reference", "metric": metric, "value": v, "unit": "SSA/s", "n_gpus": a.gpus,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                "cpu_baseline": {"value": v, "unit": "SSA/s", "cores": steps[0]["cores"], "kind": steps[0]["kind"],
                                 "sample": steps[0]["sample"]},
                "e2e": {"value": v, "unit": "SSA/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch

    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    try:
        import ssa_gpu
    except ImportError:
        import build as ssa_build
        ssa_build.build()
        import ssa_gpu

    dev = device_steps(ssa_gpu, torch, a, rank, world)
    line = {"metric": metric, "value": dev["value"], "unit": "SSA/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": dev["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 (FP64 Gram/Cholesky/Rayleigh-Ritz/LRF)", "data": "synthetic",
            "config": cfg, "gpu_launches": dev["launches"], "kernel_share": dev["share"],
            "roofline": dev["roofline"], "roofline_elem_recon": dev["roofline_elem_recon"], "clocks": dev["clocks"],
            "value_what": f"series/s of the uneven-batch pipeline (ssa_rbatch_run_device) over {a.batch} stream "
                          f"decompositions per step (mean N {dev['mean_N']:.0f}), each with the outputs of its "
                          "request type in the stream's 50:20 ratio: decompose + reconstruct -> sigma and groups "
                          "[0],[1,2]; decompose + W-correlation -> sigma, all elementary reconstructions and W "
                          "(and the groups); inputs resident in HBM"}
    if not a.no_e2e:
        line.update(server_runs(ssa_gpu, torch, a, rank, world))
    if rank == 0 and world == 1 and not a.no_plain:
        plain_path(ssa_gpu, a, n=8)  # warm-up: library, pool and recycled contexts in place
        line["plain_gpu_path"] = plain_path(ssa_gpu, a)
        line["plain_gpu_path_fresh_contexts"] = plain_path(ssa_gpu, a, recycle=False)
        if "e2e" in line:
            line["e2e_over_plain"] = line["e2e"]["value"] / line["plain_gpu_path"]["value"]
    if rank == 0 and world == 1 and not a.no_uniform:
        line["uniform_batch"] = uniform_batch(ssa_gpu, torch, a)
        line["wcorr_gram_variants"] = wgram_variants(ssa_gpu, a)
    if rank == 0 and world == 1 and not a.no_config4:
        line["config4"] = config4(ssa_gpu, torch, a)
    if rank == 0 and world == 1 and not a.no_cpu:
        line["cpu_baseline"] = cpu_reference(a, budget_s=20.0)
    acc_jobs, fc_jobs = dev.pop("acc_jobs", []), line.pop("fc_jobs", [])
    if rank == 0 and (acc_jobs or fc_jobs):
        with mp.get_context("spawn").Pool(min(len(os.sched_getaffinity(0)), 32), initializer=_pin_blas) as pool:
            rows = pool.map(_accuracy_worker, acc_jobs, chunksize=1)
            fcs = pool.map(_forecast_worker, fc_jobs, chunksize=1)
        line["accuracy"] = summarize_accuracy(rows, fcs)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
