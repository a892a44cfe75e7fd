"""ssa_wcorr_noalloc: the W-correlation entry point that allocates no device memory.

It serves callers that cannot have device memory allocated for them (an application whose
device memory is owned by another framework's allocator, or a loop that cannot afford the
synchronisation of cudaMalloc). The test calls it through the C ABI with device inputs the test
owns, twice in a row on two different decompositions, on a stream of the caller's, and checks
each result against the W-correlation of the same decomposition from the existing entry point
ssa_opt_wcorr_matrix, within the W-correlation tolerance of the parity tests; after the first
calls (which do the device's one-time set-up) a second round of calls must leave the device's
free memory unchanged. This file is collected last so that a failure here leaves every other
test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W_TOL = 1e-5


@pytest.fixture(scope="module")
def gpu():
    import ssa_gpu

    f = ssa_gpu._lib.ssa_wcorr_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    return ssa_gpu


def _reference_and_inputs(gpu, oracle, seed, N, L, k):
    import torch

    x = oracle.config2_batch(1, seed=seed, N=N)[0]
    s = gpu.SSA(x, L)
    s.decompose(k, oversampling=8, power_iters=1)
    W_ref = s.wcorr_matrix()  # existing entry point (ssa_opt_wcorr_matrix)
    U, V, sig = s.factors()
    return W_ref, _colmajor(U), _colmajor(V), torch.tensor(sig, dtype=torch.float64).cuda()


def _colmajor(A):
    """Device copy of the m x k matrix A, column-major with an even leading dimension: row j of
    the returned (k x ld) tensor is column j of A."""
    import torch

    m, k = A.shape
    ld = m + (m & 1)
    t = torch.zeros((k, ld), dtype=torch.float32)
    t[:, :m] = torch.from_numpy(np.ascontiguousarray(A.T)).float()
    return t.cuda()


def _calls(gpu, cases, prepared, stream):
    """One call per case, back to back on `stream`; returns [(W_ref, device W)]."""
    import torch

    outs = []
    for (seed, N, L, k), (W_ref, dU, dV, dS) in zip(cases, prepared):
        dW = torch.full((k, k), float("nan"), dtype=torch.float64, device="cuda")
        rc = gpu._lib.ssa_wcorr_noalloc(dU.data_ptr(), dU.shape[1], dV.data_ptr(), dV.shape[1], dS.data_ptr(),
                                        N, L, k, dW.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        outs.append((W_ref, dW))
    return outs


def _check(outs):
    for W_ref, dW in outs:
        W = dW.cpu().numpy()
        assert np.all(np.isfinite(W))
        assert np.max(np.abs(W - W_ref)) <= W_TOL
        assert np.max(np.abs(np.diag(W) - 1.0)) < 1e-6


def test_noalloc_matches_existing_entry_point_twice(gpu, oracle):
    import torch

    cases = [(11, 4000, 1000, 20), (12, 6000, 1500, 24)]
    prepared = [_reference_and_inputs(gpu, oracle, *c) for c in cases]
    stream = torch.cuda.Stream()
    # the inputs were written on torch's current stream: order the caller's stream after them
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        first = _calls(gpu, cases, prepared, stream)
    stream.synchronize()
    _check(first)
    # the first calls did the device's set-up; further calls allocate nothing: the device's free
    # memory is unchanged (output buffers are made before the measurement)
    outs = [torch.full((k, k), float("nan"), dtype=torch.float64, device="cuda") for (_, _, _, k) in cases]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for (seed, N, L, k), (W_ref, dU, dV, dS), dW in zip(cases, prepared, outs):
        rc = gpu._lib.ssa_wcorr_noalloc(dU.data_ptr(), dU.shape[1], dV.data_ptr(), dV.shape[1], dS.data_ptr(),
                                        N, L, k, dW.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
    stream.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 >= free0, (free0, free1)
    _check([(p[0], dW) for p, dW in zip(prepared, outs)])


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    import torch

    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = d.data_ptr()
    # N above the fixed maximum (8192) and k above the maximum (32): -2, nothing launched
    assert gpu._lib.ssa_wcorr_noalloc(p, 3000, p, 7002, p, 10000, 3000, 8, p, None) == -2
    assert gpu._lib.ssa_wcorr_noalloc(p, 1000, p, 3002, p, 4000, 1000, 40, p, None) == -2
    # invalid arguments: -1
    assert gpu._lib.ssa_wcorr_noalloc(p, 1000, p, 3001, p, 4000, 1000, 8, p, None) == -1  # odd ldV
    assert gpu._lib.ssa_wcorr_noalloc(None, 1000, p, 3002, p, 4000, 1000, 8, p, None) == -1
