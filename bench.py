"""Throughput benchmark of the B200 SSA hot path.

Workload (default): the uniform batch — B = 4096 independent series, N = 10000, L = 2500,
k = 50, oversampling p = 10, q = 2 power iterations; per series: randomized decomposition
(device-generated Gaussian test matrix), all k elementary reconstructions, the k x k
W-correlation matrix and the reconstructions of groups [0] and [1, 2]. One step = one pass of
that pipeline over the whole batch. Signals: seeded synthetic trend + two sinusoids (periods
U[6, 200], amplitudes U(0.5, 3)) + Gaussian noise at SNR U(0, 15) dB.

Output: one JSON line (rank 0). `value` = series per second over all ranks with inputs
resident in HBM (inputs of 328 MB per GPU are larger than L2, so no flush is needed);
`e2e` = the same through the host-buffer C ABI (ssa_batch_run: pinned host input -> device ->
pinned host outputs). `--impl reference` times the reference's CPU implementation instead.
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

import numpy as np

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
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--N", type=int, default=10000)
    ap.add_argument("--L", type=int, default=2500)
    ap.add_argument("--k", type=int, default=50)
    ap.add_argument("--p", type=int, default=10)
    ap.add_argument("--q", type=int, default=2)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    return ap.parse_args()


def workload_config(a) -> dict:
    return {"workload": f"uniform batch: {a.batch} series x N={a.N}, L={a.L}, k={a.k}, p={a.p}, q={a.q}; "
                        "decompose + all k elementary reconstructions + W-correlation + groups [0],[1,2]",
            "series_per_gpu": a.batch, "N": a.N, "L": a.L, "k": a.k, "oversampling": a.p, "power_iters": a.q,
            "l2": "inputs larger than L2 (B x N doubles per GPU)", "parallelism": "series sharded per GPU, no collective"}


def make_signals(B: int, N: int, seed: int) -> np.ndarray:
    import ssa_oracle

    return ssa_oracle.config2_batch(B, seed=seed, N=N)


# ------------------------------------------------------------------------------------------
# CPU reference leg (rank 0 only): MKL/ssa_opt_ref.h compiled from the reference (oracle/_ref)
# when present, else the NumPy FP64 port of the reference algorithm.
# ------------------------------------------------------------------------------------------

def _ref_worker(args):
    x, L, k, p = args
    import ctypes
    so = ORACLE / "_ref" / "libssa_ref.so"
    lib = ctypes.CDLL(str(so))
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    lib.refdrv_default_state.restype = ctypes.c_uint64
    lib.refdrv_pipeline.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                    ip, ip, ctypes.c_int, dp, dp, dp]
    N = len(x)
    x = np.ascontiguousarray(x, dtype=np.float64)
    groups = np.array([0, 1, 2], dtype=np.int32)
    sizes = np.array([1, 2], dtype=np.int32)
    sig = np.zeros(k)
    rec = np.zeros(2 * N)
    W = np.zeros(k * k)
    t0 = time.perf_counter()
    lib.refdrv_pipeline(x.ctypes.data_as(dp), N, L, k, p, lib.refdrv_default_state(), groups.ctypes.data_as(ip),
                        sizes.ctypes.data_as(ip), 2, sig.ctypes.data_as(dp), rec.ctypes.data_as(dp),
                        W.ctypes.data_as(dp))
    return time.perf_counter() - t0


def _port_worker(args):
    x, L, k, p, q = args
    import ssa_oracle as O
    N = len(x)
    rng = np.random.default_rng(0)
    t0 = time.perf_counter()
    Om = O.gaussian_omega(rng, N - L + 1, min(k + p, L, N - L + 1))
    d = O.decompose_randomized(x, L, k, p, Om, q=q)
    O.reconstruct(d, [0], N, L)
    O.reconstruct(d, [1, 2], N, L)
    O.wcorr_matrix(d, N, L)
    return time.perf_counter() - t0


def cpu_reference(a, budget_s: float = 20.0, series: int | None = None) -> dict:
    """Time the reference CPU path on a bounded sample: one series per process on every host
    core. Returns {"value" (series/s), "cores", "kind", "sample"}."""
    cores = len(os.sched_getaffinity(0))
    use_ref = (ORACLE / "_ref" / "libssa_ref.so").exists()
    X = make_signals(max(cores, 1) * 64, a.N, a.seed + 1000)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_pin_blas) as pool:
        # one calibration series per core, then as many rounds as fit the budget
        if use_ref:
            t = pool.map(_ref_worker, [(X[i], a.L, a.k, a.p) for i in range(cores)])
        else:
            t = pool.map(_port_worker, [(X[i], a.L, a.k, a.p, a.q) for i in range(cores)])
        per = max(statistics.median(t), 1e-6)
        rounds = max(1, int(budget_s / per)) if series is None else max(1, math.ceil(series / cores))
        n = min(rounds * cores, len(X))
        t0 = time.perf_counter()
        if use_ref:
            pool.map(_ref_worker, [(X[i], a.L, a.k, a.p) for i in range(n)])
        else:
            pool.map(_port_worker, [(X[i], a.L, a.k, a.p, a.q) for i in range(n)])
        el = time.perf_counter() - t0
    kind = "reference" if use_ref else "port"
    what = ("MKL/ssa_opt_ref.h (reference pure-C path: randomized SVD q=0, reconstruct, W-corr)" if use_ref
            else "NumPy FP64 port of MKL/ssa_opt.h randomized SVD (q as configured), reconstruct, W-corr")
    return {"value": n / el, "unit": "SSA/s", "cores": cores, "kind": kind,
            "sample": f"{n} series of N={a.N}, L={a.L}, k={a.k}, p={a.p}, one per process on {cores} cores; {what}"}


def _pin_blas():
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"


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

def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    metric = "SSA/sec"
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

    B, N = a.batch, a.N
    X = make_signals(B, N, a.seed + 7919 * rank)
    d_x = torch.from_numpy(X).to("cuda")
    batch = ssa_gpu.SSABatch(B, N, a.L, a.k, oversampling=a.p, power_iters=a.q, groups=[[0], [1, 2]])
    res = batch.device_results()
    stream = torch.cuda.ExternalStream(res["stream"])

    for w in range(a.warmup):
        batch.run_device(d_x.data_ptr(), B, seed=1000 + w)
        batch.sync()

    batch.set_profiling(True)
    launches0 = ssa_gpu.kernel_launches()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    with ClockSampler(torch.cuda.current_device()) as clk:
        ev[0].record(stream)
        for i in range(a.steps):
            batch.run_device(d_x.data_ptr(), B, seed=i)
            ev[i + 1].record(stream)
        torch.cuda.synchronize()
        batch.sync()
    launches = ssa_gpu.kernel_launches() - launches0
    prof = batch.profile()
    batch.set_profiling(False)
    step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(a.steps)]
    total_ms = ev[0].elapsed_time(ev[a.steps])
    if world > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = B * a.steps * world / (total_ms / 1e3)

    # roofline of the dominant kernel (the correlation matvec sweeps)
    K = N - a.L + 1
    kp = min(a.k + a.p, a.L, K)
    corr_ms, corr_n = prof["corr"]
    sweeps = 2 * a.q + 2  # Y = H Omega, q x (H^T Q, H Z), B = H^T Q
    # algorithmic bytes of one sweep: every probe column read once (not for the generated
    # Omega) and written once, FP32; H has N values per series.
    fwd = kp * a.L * 4
    adj = kp * K * 4
    bytes_total = B * ((0 + fwd) + a.q * ((fwd + adj) + (adj + fwd)) + (fwd + adj))
    per_launch_bytes = bytes_total / sweeps
    avg_ms = corr_ms / max(corr_n, 1)
    peak, peak_kind = measured_peak_hbm()
    achieved = per_launch_bytes / (avg_ms / 1e3) / 1e9
    dominant = max(prof.items(), key=lambda kv: kv[1][0])
    # DRAM bytes per k_corr launch from the ncu capture of the 512-series case of this shape
    # (mean over one pipeline pass: 1057.2 MB per 512 series), scaled by the series count.
    traffic = None
    if (N, a.L, a.k, a.p, a.q) == (10000, 2500, 50, 10, 2):
        traffic = 1057.2e6 / 512 * B
    roofline = {"bound": "hbm", "kernel": "k_corr (FFT correlation matvec sweep)", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": traffic, "traffic_source": "ncu dram__bytes_read+write of a 512-series capture, scaled", "avg_launch_ms": avg_ms, "algorithmic_bytes_per_launch": per_launch_bytes,
                "dominant_kernel_by_time": dominant[0]}
    share = {k: round(v[0] / max(sum(x[0] for x in prof.values()), 1e-9), 4) for k, v in prof.items() if v[1]}

    line = {"metric": metric, "value": value, "unit": "SSA/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": total_ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 (FP64 Gram/Cholesky/Rayleigh-Ritz)", "data": "synthetic",
            "config": cfg, "latency_ms": {"p50": statistics.median(step_ms),
                                          "p99": float(np.percentile(step_ms, 99)),
                                          "what": "per-step (whole batch) device time"},
            "gpu_launches": launches, "kernel_share": share, "roofline": roofline, "clocks": clk.summary()}

    if not a.no_e2e:
        xs = torch.from_numpy(X).pin_memory()
        k = batch.k
        sig = torch.empty((B, k), dtype=torch.float64).pin_memory()
        W = torch.empty((B, k, k), dtype=torch.float64).pin_memory()
        G = torch.empty((B, 2, N), dtype=torch.float64).pin_memory()
        batch.run_host_ptrs(xs.data_ptr(), B, 77, sig.data_ptr(), W.data_ptr(), G.data_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2e_steps = max(1, min(a.steps, 3))
        e0.record(stream)
        for i in range(e2e_steps):
            batch.run_host_ptrs(xs.data_ptr(), B, 77 + i, sig.data_ptr(), W.data_ptr(), G.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([e_ms], device="cuda", dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e_ms = float(t.item())
        line["e2e"] = {"value": B * e2e_steps * world / (e_ms / 1e3), "unit": "SSA/s",
                       "h2d_bytes_per_step": B * N * 8, "d2h_bytes_per_step": B * (k + k * k + 2 * N) * 8,
                       "what": "ssa_batch_run on pinned host buffers (H2D signals, D2H sigma, W, groups)"}

    if rank == 0 and world == 1 and not a.no_plain:
        # plain drop-in path: one series per call through the reference-compatible C API
        n = 16
        Xp = X[:n]
        t0 = time.perf_counter()
        for i in range(n):
            s = ssa_gpu.SSA(Xp[i], a.L)
            s.decompose(a.k, oversampling=a.p, power_iters=a.q)
            s.reconstruct([0])
            s.reconstruct([1, 2])
            s.wcorr_matrix()
            del s
        el = time.perf_counter() - t0
        line["plain_gpu_path"] = {"value": n / el, "unit": "SSA/s",
                                  "what": f"{n} series, one per call: SSA() + decompose(q={a.q}) + 2 reconstructs + "
                                          "wcorr_matrix through libssa.so (host wall clock)"}
    if rank == 0 and world == 1 and not a.no_cpu:
        line["cpu_baseline"] = cpu_reference(a, budget_s=20.0)

    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
