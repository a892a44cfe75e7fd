"""CPU checks of the drop-in boundary: libssa.so loads without a GPU, exports every function
declared in include/*.h and the export list of the reference shared library, and the unchanged
reference ctypes wrapper binds against it. No device calls are made here (the one compute call
is the host eigen-solver)."""
import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "singular-spectrum-analysis_b200" / "libssa.so"

# Export list of the reference shared library (MKL/py/ssa.def) and the names its ctypes
# wrapper binds unconditionally (MKL/py/ssa_wrapper.py:125-204, 272-291).
REFERENCE_EXPORTS = """
ssa_opt_init ssa_opt_decompose ssa_opt_decompose_block ssa_opt_decompose_randomized ssa_opt_reconstruct
ssa_opt_forecast ssa_opt_forecast_full ssa_opt_forecast_with_lrf ssa_opt_compute_lrf ssa_opt_lrf_free
ssa_opt_wcorr_matrix ssa_opt_wcorr_pair ssa_opt_variance_explained ssa_opt_find_periodic_pairs
ssa_opt_component_stats ssa_opt_component_stats_free ssa_opt_get_trend ssa_opt_get_noise ssa_opt_cache_ffts
ssa_opt_free mssa_opt_init mssa_opt_decompose mssa_opt_reconstruct mssa_opt_reconstruct_all
mssa_opt_series_contributions mssa_opt_variance_explained mssa_opt_free ssa_opt_extend
ssa_opt_get_singular_values ssa_opt_get_eigenvalues ssa_opt_get_total_variance ssa_opt_prepare
ssa_opt_update_signal ssa_opt_free_prepared ssa_opt_vforecast ssa_opt_vforecast_full ssa_opt_vforecast_fast
ssa_opt_cadzow ssa_opt_cadzow_weighted ssa_opt_cadzow_inplace ssa_opt_parestimate ssa_opt_parestimate_free
ssa_opt_gapfill ssa_opt_gapfill_simple ssa_mkl_init ssa_mkl_init_14900kf ssa_mkl_init_generic
ssa_mkl_set_threads ssa_mkl_get_threads ssa_mkl_get_cpu_info ssa_mkl_disable_affinity
""".split()


@pytest.fixture(scope="module")
def lib():
    if not LIB.exists():
        import importlib.util
        spec = importlib.util.spec_from_file_location("ssabuild", ROOT / "singular-spectrum-analysis_b200" / "build.py")
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        m.build()
    return ctypes.CDLL(str(LIB))


def _declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w \*]*?\b([a-z][a-z0-9_]+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return {n for n in names if n.startswith(("ssa_", "mssa_"))}


def test_exports_every_declared_function(lib):
    declared = _declared_functions()
    assert len(declared) > 50
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_exports_reference_symbols(lib):
    missing = [n for n in REFERENCE_EXPORTS if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_fits_ctypes_buffer(lib):
    lib.ssa_b200_sizeof_ssa_opt.restype = ctypes.c_int
    assert lib.ssa_b200_sizeof_ssa_opt() <= 1024


def test_built_for_sm100a_only():
    out = subprocess.run(["cuobjdump", "--list-elf", str(LIB)], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def _reference_wrapper():
    from conftest import reference_dir

    d = reference_dir()
    w = d / "py" / "ssa_wrapper.py" if d is not None else None
    if w is None or not w.exists():
        pytest.skip("reference wrapper not present on this machine")
    return w


def test_unchanged_reference_wrapper_binds(lib):
    REF_WRAPPER = _reference_wrapper()
    code = (
        "import importlib.util\n"
        f"spec = importlib.util.spec_from_file_location('ssa_wrapper', r'{REF_WRAPPER}')\n"
        "m = importlib.util.module_from_spec(spec); spec.loader.exec_module(m)\n"
        "assert m._HAS_GETTERS and m._HAS_CADZOW and m._HAS_ESPRIT and m._HAS_GAPFILL and m._HAS_VFORECAST\n"
        "print('ok')\n"
    )
    import os, sys
    env = dict(os.environ, LD_LIBRARY_PATH=str(LIB.parent))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr


def test_host_eigen_solver_vs_numpy():
    """ssa_b200_eigvals (the ESPRIT eigen-solver: Hessenberg + Francis double-shift QR) against
    numpy on random, rotation-block, companion and defective matrices; no GPU call."""
    import ssa_gpu

    rng = np.random.default_rng(3)
    cases = [rng.standard_normal((n, n)) for n in (1, 2, 3, 5, 8, 17, 40, 64)]
    th = [0.1, 0.7, 2.0]
    R = np.zeros((6, 6))
    for i, t in enumerate(th):
        c, s = np.cos(t), np.sin(t)
        R[2 * i:2 * i + 2, 2 * i:2 * i + 2] = [[c, -s], [s, c]]
    Q = np.linalg.qr(rng.standard_normal((6, 6)))[0]
    cases.append(Q @ R @ Q.T)  # eigenvalues on the unit circle
    comp = np.zeros((7, 7))
    comp[0, :] = -np.poly(np.arange(1, 8))[1:]
    comp[1:, :-1] = np.eye(6)
    cases.append(comp)  # companion matrix, roots 1..7
    cases.append(np.array([[2.0, 1.0], [0.0, 2.0]]))  # defective
    for A in cases:
        got = np.sort_complex(ssa_gpu.eigvals(A))
        ref = np.sort_complex(np.linalg.eigvals(A))
        scale = max(1.0, np.abs(ref).max())
        assert np.max(np.abs(got - ref)) <= 1e-8 * scale, (A.shape, np.max(np.abs(got - ref)))


def test_fft_size_codes():
    """FFT lengths of the uneven batches: powers of two, and 49152 / 81920 / 98304 between the
    cluster powers of two (ssa_b200_fft_length)."""
    import ssa_gpu

    f = ssa_gpu._lib.ssa_b200_fft_length
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int]
    cases = {500: 512, 32768: 32768, 32769: 49152, 49152: 49152, 49153: 65536, 65536: 65536,
             65537: 81920, 81920: 81920, 81921: 98304, 98304: 98304, 98305: 131072, 131072: 131072}
    for N, M in cases.items():
        assert f(N) == M, (N, f(N))
    assert f(131073) == -1 and f(0) == -1
