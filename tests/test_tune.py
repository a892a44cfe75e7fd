"""The autotuner's table (ssa_b200_tune_set / ssa_tune): host-side round trip and validation on
the CPU; on the GPU a small tuning run applies a table under which results still meet the
parity tolerances."""
import json

import numpy as np
import pytest


@pytest.fixture(scope="module")
def tune():
    import ssa_tune

    return ssa_tune


def test_table_round_trip_and_validation(tune):
    before = tune.current()
    try:
        g = [0] * tune.NCODES
        g[13], g[15] = 592, 2368
        tune.apply({"gram_ctas": g, "multi": False, "multi_ctas_per_sm": 1})
        cur = tune.current()
        assert cur["gram_ctas"] == g and cur["multi"] is False and cur["multi_ctas_per_sm"] == 1
        with pytest.raises(ValueError):
            tune.apply({"gram_ctas": [-1] * tune.NCODES, "multi": True, "multi_ctas_per_sm": 0})
        with pytest.raises(ValueError):
            tune.apply({"gram_ctas": g, "multi": True, "multi_ctas_per_sm": 3})
    finally:
        tune.apply(before)
    assert tune.current() == before


def test_size_codes(tune):
    assert tune.size_code(1000) == 9 and tune.size_code(16384) == 13 and tune.size_code(16385) == 14
    assert tune.size_code(40000) == 17 and tune.size_code(60000) == 15 and tune.size_code(90000) == 18
    assert tune.size_code(70000) == 19 and tune.size_code(81920) == 19 and tune.size_code(81921) == 18
    assert tune.size_code(131073) == -1


def test_cache_keyed_by_gpu_and_library(tune, tmp_path):
    path = tmp_path / "tune.json"
    table = {"gram_ctas": [0] * tune.NCODES, "multi": True, "multi_ctas_per_sm": 0}
    path.write_text(json.dumps({"key": tune.cache_key(), "table": table}))
    assert tune.load(path)["table"] == table
    path.write_text(json.dumps({"key": dict(tune.cache_key(), library="other"), "table": table}))
    assert tune.load(path) is None


@pytest.mark.gpu
def test_autotune_small_run_keeps_parity(tune, oracle, tmp_path):
    import ssa_gpu

    before = tune.current()
    try:
        out = tune.autotune(cache=tmp_path / "t.json", buckets=[14], series=8, reps=1, retune=True)
        assert (tmp_path / "t.json").exists() and out["table"] == tune.current()
        assert tune.load(tmp_path / "t.json")["table"] == out["table"]
        mix = oracle.config3_batch(6, seed=44, nmin=500, nmax=30000)
        xs, Ls, ks = [m[0] for m in mix], [m[1] for m in mix], [m[2] for m in mix]
        rb = ssa_gpu.SSARaggedBatch(oversampling=10, power_iters=2)
        sig, W, G = rb.run(xs, Ls, ks, seed=2)
        for s, (x, L, k) in enumerate(mix):
            N = len(x)
            K = N - L + 1
            kk, kp = oracle.clamp_kp(L, K, k, 10)
            d = oracle.decompose_randomized(x, L, kk, 10, oracle.device_gaussian(oracle.series_seed(2, s), K, kp), q=2)
            assert np.max(np.abs(sig[s][:3] - d.sigma[:3]) / d.sigma[:3]) <= 1e-5
    finally:
        tune.apply(before)
