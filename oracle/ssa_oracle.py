"""CPU oracle for the SSA decomposition / reconstruction hot path (TEST INFRASTRUCTURE ONLY).

This module is a float64 NumPy restatement of the reference algorithm of SSA-Opt
(``MKL/ssa_opt.h``). It exists to CHECK the CUDA path: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it. The product
(``libssa.so``) never calls into it and has no CPU fallback.

Every function cites the reference lines it restates. LAPACK calls of the reference are
restated with the same LAPACK routines as NumPy exposes them: ``numpy.linalg.qr`` is
``dgeqrf`` + ``dorgqr`` (ssa_opt.h:1724-1725), ``numpy.linalg.svd(full_matrices=False)`` is
``dgesdd`` with job 'S' (ssa_opt.h:1731).

Parity pinning: the restatement is checked in ``tests/test_oracle.py`` against
(a) the reference's own dependency-free C implementation ``MKL/ssa_opt_ref.h``, compiled from
its source by ``oracle/Makefile`` into ``oracle/_ref/libssa_ref.so`` (same Omega through the
reference's own xorshift/Box-Muller generator), (b) the known-answer tests of
``MKL/test/ssa_opt_test.c`` (matvec vs direct sum < 1e-10, fast vs slow W-correlation < 1e-6,
W diagonal/symmetry, variance partition), and (c) the exact dense SVD of the trajectory matrix.

Extension beyond the reference: ``q`` power iterations inside the randomized range finder
(the reference has q = 0 only, ssa_opt.h:1685-1763). With q = 0 the function is the reference.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

# ---------------------------------------------------------------------------------------------
# Dimensions and weights
# ---------------------------------------------------------------------------------------------


def next_pow2(n: int) -> int:
    """ssa_opt.h:434-440 (ssa_opt_next_pow2)."""
    p = 1
    while p < n:
        p <<= 1
    return p


def ref_fft_len(N: int, L: int) -> int:
    """FFT length the reference uses: next_pow2(N + K - 1) (ssa_opt.h:1047-1049)."""
    K = N - L + 1
    return next_pow2(N + K - 1)


def inv_diag_count(N: int, L: int) -> np.ndarray:
    """1 / min(t+1, L, K, N-t) for t < N (ssa_opt.h:1270-1279)."""
    K = N - L + 1
    t = np.arange(N)
    cnt = np.minimum(np.minimum(t + 1, L), np.minimum(K, N - t))
    return 1.0 / cnt.astype(np.float64)


def hankel(x: np.ndarray, L: int) -> np.ndarray:
    """Explicit trajectory matrix H[i, j] = x[i + j], L x K (ssa_opt.h:862-866 comment)."""
    N = len(x)
    K = N - L + 1
    idx = np.arange(L)[:, None] + np.arange(K)[None, :]
    return np.asarray(x, dtype=np.float64)[idx]


# ---------------------------------------------------------------------------------------------
# Hankel matvecs (ssa_opt.h:871-1004)
# ---------------------------------------------------------------------------------------------


def hankel_matvec(x: np.ndarray, v: np.ndarray, L: int, fft_len: Optional[int] = None) -> np.ndarray:
    """y = H v = first L of IFFT(FFT(x) * conj(FFT(v))) (ssa_opt.h:871-883).

    Columns of ``v`` (K x b) are processed like hankel_matvec_block (ssa_opt.h:910-954).
    """
    x = np.asarray(x, dtype=np.float64)
    N = len(x)
    K = N - L + 1
    M = fft_len or ref_fft_len(N, L)
    fx = np.fft.rfft(x, M)
    V = np.asarray(v, dtype=np.float64)
    one = V.ndim == 1
    if one:
        V = V[:, None]
    assert V.shape[0] == K
    fv = np.fft.rfft(V, M, axis=0)
    y = np.fft.irfft(fx[:, None] * np.conj(fv), M, axis=0)[:L]
    return y[:, 0] if one else y


def hankel_matvec_T(x: np.ndarray, u: np.ndarray, L: int, fft_len: Optional[int] = None) -> np.ndarray:
    """z = H^T u = first K of IFFT(FFT(x) * conj(FFT(u))) (ssa_opt.h:891-903, 960-1004)."""
    x = np.asarray(x, dtype=np.float64)
    N = len(x)
    K = N - L + 1
    M = fft_len or ref_fft_len(N, L)
    fx = np.fft.rfft(x, M)
    U = np.asarray(u, dtype=np.float64)
    one = U.ndim == 1
    if one:
        U = U[:, None]
    assert U.shape[0] == L
    fu = np.fft.rfft(U, M, axis=0)
    z = np.fft.irfft(fx[:, None] * np.conj(fu), M, axis=0)[:K]
    return z[:, 0] if one else z


def hankel_matvec_direct(x: np.ndarray, v: np.ndarray, L: int) -> np.ndarray:
    """Direct O(LK) sum y[i] = sum_j x[i+j] v[j] (MKL/test/ssa_opt_test.c:1482-1490)."""
    return hankel(x, L) @ np.asarray(v, dtype=np.float64)


def hankel_matvec_T_direct(x: np.ndarray, u: np.ndarray, L: int) -> np.ndarray:
    """Direct z[j] = sum_i x[i+j] u[i] (MKL/test/ssa_opt_test.c:1530-1538)."""
    return hankel(x, L).T @ np.asarray(u, dtype=np.float64)


# ---------------------------------------------------------------------------------------------
# Decompositions
# ---------------------------------------------------------------------------------------------


@dataclass
class Decomposition:
    """Result arrays with the reference layout: U is L x k (column i = U[:, i]), V is K x k."""

    U: np.ndarray
    V: np.ndarray
    sigma: np.ndarray
    eigenvalues: np.ndarray
    total_variance: float

    @property
    def k(self) -> int:
        return len(self.sigma)


def _sign_fix(U: np.ndarray, V: np.ndarray) -> None:
    """sum(U[:, i]) < 0 => negate U[:, i] and V[:, i] (ssa_opt.h:1749-1759)."""
    s = U.sum(axis=0)
    neg = s < 0
    U[:, neg] *= -1.0
    V[:, neg] *= -1.0


def clamp_kp(L: int, K: int, k: int, oversampling: int) -> tuple[int, int]:
    """p default 8, kp = min(k + p, L, K), k = min(k, kp) (ssa_opt.h:1691-1694)."""
    p = 8 if oversampling <= 0 else oversampling
    kp = min(k + p, min(L, K))
    return min(k, kp), kp


def decompose_randomized(
    x: np.ndarray,
    L: int,
    k: int,
    oversampling: int,
    Omega: np.ndarray,
    q: int = 0,
    fft_len: Optional[int] = None,
) -> Decomposition:
    """Randomized SVD of the trajectory matrix with a given Gaussian test matrix.

    Restates ssa_opt_decompose_randomized (ssa_opt.h:1685-1763):
      Y = H Omega (:1720) -> Q = qr(Y) (:1723-1725) -> B = H^T Q (:1728)
      -> gesdd(B) = B_left S B_right_T (:1731) -> U = Q B_right_T^T, V = B_left (:1736-1738)
      -> sigma, lambda, total_variance (:1741-1746) -> sign fix (:1749-1759).
    Extension: ``q`` subspace (power) iterations Z = H^T Q, Q_z = qr(Z), Y = H Q_z, Q = qr(Y)
    between the first QR and B (not in the reference; q = 0 reproduces it).
    ``Omega`` is K x kp column-major in the reference, i.e. a (K, kp) array here.
    """
    x = np.asarray(x, dtype=np.float64)
    N = len(x)
    K = N - L + 1
    k, kp = clamp_kp(L, K, k, oversampling)
    Om = np.asarray(Omega, dtype=np.float64)
    assert Om.shape[0] == K and Om.shape[1] >= kp, (Om.shape, K, kp)
    Om = Om[:, :kp]
    Y = hankel_matvec(x, Om, L, fft_len)
    Q, _ = np.linalg.qr(Y, mode="reduced")
    for _ in range(q):
        Z = hankel_matvec_T(x, Q, L, fft_len)
        Qz, _ = np.linalg.qr(Z, mode="reduced")
        Y = hankel_matvec(x, Qz, L, fft_len)
        Q, _ = np.linalg.qr(Y, mode="reduced")
    B = hankel_matvec_T(x, Q, L, fft_len)
    B_left, S, B_right_T = np.linalg.svd(B, full_matrices=False)
    U = Q @ B_right_T.T[:, :k]
    V = B_left[:, :k].copy()
    sigma = S[:k].copy()
    lam = sigma * sigma
    _sign_fix(U, V)
    return Decomposition(U, V, sigma, lam, float(lam.sum()))


def decompose_block(
    x: np.ndarray,
    L: int,
    k: int,
    block_size: int,
    max_iter: int,
    V0_blocks: Sequence[np.ndarray],
    fft_len: Optional[int] = None,
) -> Decomposition:
    """Block power iteration with Rayleigh-Ritz (ssa_opt_decompose_block, ssa_opt.h:1765-1933).

    ``V0_blocks[i]`` is the K x cur_b uniform(-0.5, 0.5) start block that the reference draws
    from its RNG at :1813 for the i-th block.
    """
    x = np.asarray(x, dtype=np.float64)
    N = len(x)
    K = N - L + 1
    b = min(block_size, min(k, min(L, K)))
    k = min(k, min(L, K))
    U = np.zeros((L, k))
    V = np.zeros((K, k))
    sig = np.zeros(k)
    comp = 0
    blk = 0
    QR_INTERVAL = 5  # ssa_opt.h:1821

    def qr(A):
        return np.linalg.qr(A, mode="reduced")[0]

    while comp < k:
        cur_b = min(b, k - comp)
        Vb = np.asarray(V0_blocks[blk], dtype=np.float64)[:, :cur_b].copy()
        blk += 1
        if comp > 0:  # :1814-1818 deflation against earlier V
            Vb -= V[:, :comp] @ (V[:, :comp].T @ Vb)
        Vb = qr(Vb)  # :1819-1820
        Ub = None
        for it in range(max_iter):  # :1822-1846
            Ub = hankel_matvec(x, Vb, L, fft_len)
            if comp > 0:
                Ub -= U[:, :comp] @ (U[:, :comp].T @ Ub)
            if (it % QR_INTERVAL == 0) or (it == max_iter - 1):
                Ub = qr(Ub)
            Vb = hankel_matvec_T(x, Ub, L, fft_len)
            if comp > 0:
                Vb -= V[:, :comp] @ (V[:, :comp].T @ Vb)
            if (it > 0 and it % QR_INTERVAL == 0) or (it == max_iter - 1):
                Vb = qr(Vb)
        U2 = hankel_matvec(x, Vb, L, fft_len)  # :1847
        if comp > 0:
            U2 -= U[:, :comp] @ (U[:, :comp].T @ U2)
        Msmall = Ub.T @ U2  # :1853
        Us, Ss, Vts = np.linalg.svd(Msmall)  # :1854 (gesvd 'A','A')
        U2 = Ub @ Us  # :1867
        W = Vb @ Vts.T  # :1868
        sig[comp:comp + cur_b] = Ss
        U[:, comp:comp + cur_b] = U2
        V[:, comp:comp + cur_b] = W
        Vb = hankel_matvec_T(x, U[:, comp:comp + cur_b], L, fft_len)  # :1878-1880
        if comp > 0:
            Vb -= V[:, :comp] @ (V[:, :comp].T @ Vb)
        for i in range(cur_b):  # :1886-1893
            s = sig[comp + i]
            col = Vb[:, i] / s if s > 1e-12 else Vb[:, i]
            V[:, comp + i] = col
        comp += cur_b
    # selection sort by sigma descending (:1896-1908), stable w.r.t. the reference swap order
    for i in range(k - 1):
        for j in range(i + 1, k):
            if sig[j] > sig[i]:
                sig[[i, j]] = sig[[j, i]]
                U[:, [i, j]] = U[:, [j, i]]
                V[:, [i, j]] = V[:, [j, i]]
    _sign_fix(U, V)
    lam = sig * sig
    return Decomposition(U, V, sig, lam, float(lam.sum()))


def dense_svd(x: np.ndarray, L: int, k: int) -> Decomposition:
    """Truth oracle: exact dense SVD of the L x K trajectory matrix, reference sign rule."""
    H = hankel(x, L)
    Uf, S, Vt = np.linalg.svd(H, full_matrices=False)
    U = Uf[:, :k].copy()
    V = Vt[:k].T.copy()
    _sign_fix(U, V)
    lam = S[:k] ** 2
    return Decomposition(U, V, S[:k].copy(), lam, float(lam.sum()))


# ---------------------------------------------------------------------------------------------
# Reconstruction and W-correlation
# ---------------------------------------------------------------------------------------------


def reconstruct(dec: Decomposition, group: Sequence[int], N: int, L: int,
                fft_len: Optional[int] = None) -> np.ndarray:
    """x~ = inv_w * IFFT(sum_{i in g} FFT(sigma_i u_i) * FFT(v_i)) (ssa_opt.h:2325-2400).

    Indices outside [0, k) are skipped (:2347-2348). An empty group is an error (:2327).
    """
    if len(group) < 1:
        raise ValueError("empty group")
    M = fft_len or ref_fft_len(N, L)
    acc = np.zeros(M // 2 + 1, dtype=np.complex128)
    for idx in group:
        if idx < 0 or idx >= dec.k:
            continue
        acc += np.fft.rfft(dec.sigma[idx] * dec.U[:, idx], M) * np.fft.rfft(dec.V[:, idx], M)
    return np.fft.irfft(acc, M)[:N] * inv_diag_count(N, L)


def reconstruct_direct(dec: Decomposition, group: Sequence[int], N: int, L: int) -> np.ndarray:
    """Anti-diagonal averaging of sum_{i in g} sigma_i u_i v_i^T, computed by explicit sums."""
    K = N - L + 1
    X = np.zeros((L, K))
    for idx in group:
        if 0 <= idx < dec.k:
            X += dec.sigma[idx] * np.outer(dec.U[:, idx], dec.V[:, idx])
    out = np.zeros(N)
    for d in range(N):
        i0 = max(0, d - (K - 1))
        i1 = min(L - 1, d)
        ii = np.arange(i0, i1 + 1)
        out[d] = X[ii, d - ii].mean()
    return out


def elementary_reconstructions(dec: Decomposition, N: int, L: int) -> np.ndarray:
    """All k elementary reconstructions, k x N (row i = reconstruct([i]))."""
    return np.stack([reconstruct(dec, [i], N, L) for i in range(dec.k)])


def wcorr_matrix(dec: Decomposition, N: int, L: int, fft_len: Optional[int] = None) -> np.ndarray:
    """W-correlation matrix, k x k row-major (ssa_opt_wcorr_matrix, ssa_opt.h:2407-2484).

    h_i = IFFT(FFT(u_i) FFT(v_i)); ||h_i||_w^2 = sigma_i^2 sum h_i^2 inv_w (:2466-2468);
    G_i = (sigma_i / ||h_i||_w) h_i sqrt(inv_w) (:2469-2471), zero row when the norm <= 1e-12;
    W = G G^T (:2473), mirrored (:2474-2476).
    """
    M = fft_len or ref_fft_len(N, L)
    iw = inv_diag_count(N, L)
    siw = np.sqrt(iw)
    k = dec.k
    G = np.zeros((k, N))
    for i in range(k):
        h = np.fft.irfft(np.fft.rfft(dec.U[:, i], M) * np.fft.rfft(dec.V[:, i], M), M)[:N]
        s = dec.sigma[i]
        nrm = math.sqrt(float(np.sum(h * h * iw)) * s * s)
        scale = s / nrm if nrm > 1e-12 else 0.0
        G[i] = scale * h * siw
    W = G @ G.T
    iu = np.triu_indices(k, 1)
    W[(iu[1], iu[0])] = W[iu]
    return W


def wcorr_pair(dec: Decomposition, N: int, L: int, i: int, j: int) -> float:
    """ssa_opt_wcorr_pair (ssa_opt.h:2551-2632); 0.0 for out-of-range indices."""
    if i < 0 or j < 0 or i >= dec.k or j >= dec.k:
        return 0.0
    M = ref_fft_len(N, L)
    iw = inv_diag_count(N, L)
    hi = np.fft.irfft(np.fft.rfft(dec.U[:, i], M) * np.fft.rfft(dec.V[:, i], M), M)[:N]
    hj = np.fft.irfft(np.fft.rfft(dec.U[:, j], M) * np.fft.rfft(dec.V[:, j], M), M)[:N]
    si, sj = dec.sigma[i], dec.sigma[j]
    inner = float(np.sum(hi * hj * iw)) * si * sj
    ni = float(np.sum(hi * hi * iw)) * si * si
    nj = float(np.sum(hj * hj * iw)) * sj * sj
    den = math.sqrt(ni) * math.sqrt(nj)
    return inner / den if den > 1e-12 else 0.0


# ---------------------------------------------------------------------------------------------
# LRF / R-forecast (ssa_opt.h:2766-2885) and getters (ssa_opt.h:3086-3145)
# ---------------------------------------------------------------------------------------------


def compute_lrf(dec: Decomposition, group: Sequence[int], L: int) -> tuple[np.ndarray, float]:
    """pi_g = U[L-1, g]; nu^2 = sum pi^2; invalid if nu^2 >= 1 - 1e-10;
    R[j] = sum_g pi_g U[j, g] / (1 - nu^2), j < L - 1 (ssa_opt.h:2766-2816).
    Raises ValueError where the reference returns -1."""
    if len(group) < 1:
        raise ValueError("empty group")
    for idx in group:
        if idx < 0 or idx >= dec.k:
            raise ValueError("group index out of range")
    g = np.asarray(group, dtype=np.int64)
    pi = dec.U[L - 1, g]
    nu2 = float(np.sum(pi * pi))
    if nu2 >= 1.0 - 1e-10:
        raise ValueError("verticality >= 1")
    R = (dec.U[: L - 1, g] @ pi) / (1.0 - nu2)
    return R, nu2


def forecast_with_lrf(R: np.ndarray, base: np.ndarray, n_forecast: int) -> np.ndarray:
    """Recurrence x[n] = sum_j R[j] buf[h + j] over the last L-1 values (ssa_opt.h:2818-2841)."""
    w = len(R)
    buf = np.zeros(w + n_forecast)
    buf[:w] = base[len(base) - w:]
    out = np.zeros(n_forecast)
    for h in range(n_forecast):
        f = 0.0
        for j in range(w):
            f += R[j] * buf[h + j]
        buf[w + h] = f
        out[h] = f
    return out


def forecast(dec: Decomposition, group: Sequence[int], n_forecast: int, N: int, L: int) -> np.ndarray:
    """ssa_opt_forecast (ssa_opt.h:2843-2867)."""
    R, _ = compute_lrf(dec, group, L)
    rec = reconstruct(dec, group, N, L)
    return forecast_with_lrf(R, rec, n_forecast)


def forecast_full(dec: Decomposition, group: Sequence[int], n_forecast: int, N: int, L: int) -> np.ndarray:
    """ssa_opt_forecast_full (ssa_opt.h:2869-2885): reconstruction followed by the forecast."""
    R, _ = compute_lrf(dec, group, L)
    rec = reconstruct(dec, group, N, L)
    return np.concatenate([rec, forecast_with_lrf(R, rec, n_forecast)])


def _vforecast_steps(dec: Decomposition, group: Sequence[int], L: int, buf: np.ndarray, n_forecast: int) -> np.ndarray:
    """V-forecast recurrence as the reference writes it (ssa_opt.h:2941-2962): every step projects
    the last L-1 values z on each group eigenvector and sums pi_g (U_trunc,g . z) / (1 - nu^2).
    `buf` holds the starting window in its first L-1 entries and receives the forecasts."""
    _, nu2 = compute_lrf(dec, group, L)  # index and verticality checks of ssa_opt.h:2912-2922
    scale = 1.0 / (1.0 - nu2)
    w = L - 1
    out = np.zeros(n_forecast)
    for h in range(n_forecast):
        z = buf[h:h + w]
        x_new = 0.0
        for idx in group:
            u = dec.U[:, idx]
            x_new += u[L - 1] * float(np.dot(u[:w], z))
        x_new *= scale
        buf[w + h] = x_new
        out[h] = x_new
    return out


def vforecast(dec: Decomposition, group: Sequence[int], n_forecast: int, N: int, L: int) -> np.ndarray:
    """ssa_opt_vforecast (ssa_opt.h:2906-2966): forecast from the group's reconstruction."""
    rec = reconstruct(dec, group, N, L)
    buf = np.zeros(L - 1 + n_forecast)
    buf[:L - 1] = rec[N - (L - 1):]
    return _vforecast_steps(dec, group, L, buf, n_forecast)


def vforecast_full(dec: Decomposition, group: Sequence[int], n_forecast: int, N: int, L: int) -> np.ndarray:
    """ssa_opt_vforecast_full (ssa_opt.h:2968-3014): reconstruction followed by the forecast."""
    rec = reconstruct(dec, group, N, L)
    return np.concatenate([rec, vforecast(dec, group, n_forecast, N, L)])


def vforecast_fast(dec: Decomposition, group: Sequence[int], base: np.ndarray, n_forecast: int, L: int) -> np.ndarray:
    """ssa_opt_vforecast_fast (ssa_opt.h:3016-3078): the recurrence from the last L-1 values of
    a given base signal (len(base) >= L - 1)."""
    if len(base) < L - 1 or n_forecast < 1:
        raise ValueError("base shorter than L - 1")
    buf = np.zeros(L - 1 + n_forecast)
    buf[:L - 1] = np.asarray(base, dtype=np.float64)[len(base) - (L - 1):]
    return _vforecast_steps(dec, group, L, buf, n_forecast)


def gap_linear_start(x: np.ndarray, gap: np.ndarray) -> None:
    """Initial fill of NaN runs by the line between their valid neighbours (ssa_opt.h:3450-3494):
    point j of a run of n at fraction (j + 1) / (n + 1) (a single point: 0.5); one neighbour
    only: its value; none: 0."""
    N = len(x)
    i = 0
    while i < N:
        if not gap[i]:
            i += 1
            continue
        a = i
        while i < N and gap[i]:
            i += 1
        n = i - a
        lv = x[a - 1] if a > 0 else (x[i] if i < N else 0.0)
        rv = x[i] if i < N else lv
        for j in range(n):
            t = (j + 1) / (n + 1) if n > 1 else 0.5
            x[a + j] = lv + t * (rv - lv)


def gapfill(x: np.ndarray, L: int, rank: int, max_iter: int, tol: float, omega_fn) -> tuple:
    """ssa_opt_gapfill (ssa_opt.h:3497-3683): linear start, then per iteration a rank-`rank`
    reconstruction (randomized, q = 0, oversampling 8, a fresh context: omega_fn(K, kp) gives
    its test matrix) written into the gaps until the relative change of the gap values < tol.
    Returns (filled signal, iterations, final_diff, converged, n_gaps); ValueError where the
    reference returns -1."""
    y = np.asarray(x, dtype=np.float64).copy()
    N = len(y)
    if N < 4 or L < 2 or L > N - 1 or rank < 1:
        raise ValueError("bad shape")
    gap = np.isnan(y)
    n_gaps = int(gap.sum())
    if n_gaps == 0:
        return y, 0, 0.0, True, 0
    if N - n_gaps < L + rank:
        raise ValueError("not enough data")
    gap_linear_start(y, gap)
    K = N - L + 1
    kp = min(rank + 8, L, K)
    Om = omega_fn(K, kp)
    old = y[gap].copy()
    diff, converged, it = 1e10, False, 0
    group = list(range(rank))
    while it < max_iter:
        dec = decompose_randomized(y, L, rank, 8, Om, q=0)
        rec = reconstruct(dec, group, N, L)
        new = rec[gap]
        y[gap] = new
        so = float(np.sum(old * old))
        sd = float(np.sum((new - old) ** 2))
        diff = math.sqrt(sd / so) if so > 1e-12 else math.sqrt(sd)
        it += 1
        if diff < tol:
            converged = True
            break
        old = new.copy()
    return y, it, diff, converged, n_gaps


def gapfill_simple(x: np.ndarray, L: int, rank: int, omega_fn) -> tuple:
    """ssa_opt_gapfill_simple (ssa_opt.h:3685-3878): each NaN run, left to right, from the
    forecast of the segment before it and the reversed segment after it (each when at least
    L + rank long; randomized q = 0, oversampling 8, fresh contexts), weighted linearly towards
    the nearer side; neither: the mean of the neighbours. A right segment that still holds a
    later run gives no forecast (the reference would decompose its NaNs). Returns (signal, n_gaps)."""
    y = np.asarray(x, dtype=np.float64).copy()
    N = len(y)
    if N < 4 or L < 2 or L > N - 1 or rank < 1:
        raise ValueError("bad shape")
    gap = np.isnan(y)
    n_gaps = int(gap.sum())
    group = list(range(rank))

    def seg_forecast(seg, h):
        n = len(seg)
        K = n - L + 1
        kp = min(rank + 8, L, K)
        dec = decompose_randomized(seg, L, rank, 8, omega_fn(K, kp), q=0)
        try:
            return forecast(dec, group[:min(rank, dec.k)], h, n, L)
        except ValueError:
            return None

    i = 0
    while i < N:
        if not gap[i]:
            i += 1
            continue
        a = i
        while i < N and gap[i]:
            i += 1
        glen = i - a
        fl = seg_forecast(y[:a].copy(), glen) if a >= L + rank else None
        right_clean = N - i >= L + rank and not gap[i:].any()  # a later unfilled run: no forecast
        fr = seg_forecast(y[::-1][:N - i].copy(), glen) if right_clean else None
        for j in range(glen):
            v = w = 0.0
            if fl is not None:
                wl = (glen - j) / glen
                v += wl * fl[j]
                w += wl
            if fr is not None:
                wr = (j + 1) / glen
                v += wr * fr[glen - 1 - j]
                w += wr
            if w > 0:
                y[a + j] = v / w
            else:
                lv = y[a - 1] if a > 0 else 0.0
                rv = y[i] if i < N else lv
                y[a + j] = 0.5 * (lv + rv)
    return y, n_gaps


def parestimate(dec: Decomposition, group, L: int) -> dict:
    """ESPRIT (ssa_opt.h:4304-4558): Z = argmin ||U_up Z - U_down|| over the selected
    eigenvectors (least squares), eigenvalues of Z -> modulus |lambda|, rate log|lambda| (-30
    below 1e-12), frequency arg(lambda) / 2 pi, period 1 / |frequency| (inf below 1e-12). The
    eigenvalues come in numpy's order; compare them as a set."""
    idx = list(range(dec.k)) if not group else list(group)
    if not idx or L < 3 or any(i < 0 or i >= dec.k for i in idx):
        raise ValueError("bad group")
    U = dec.U[:, idx]
    Z = np.linalg.lstsq(U[:L - 1], U[1:L], rcond=None)[0]
    lam = np.linalg.eigvals(Z)
    mod = np.abs(lam)
    freq = np.angle(lam) / (2 * np.pi)
    with np.errstate(divide="ignore"):
        per = np.where(np.abs(freq) > 1e-12, 1.0 / np.abs(freq), np.inf)
    rate = np.where(mod > 1e-12, np.log(np.maximum(mod, 1e-300)), -30.0)
    return {"eig": lam, "moduli": mod, "frequencies": freq, "periods": per, "rates": rate}


def variance_explained(dec: Decomposition, start: int, end: int) -> float:
    """ssa_opt_variance_explained (ssa_opt.h:3110-3120)."""
    if start < 0 or dec.total_variance <= 0:
        return 0.0
    if end < 0 or end >= dec.k:
        end = dec.k - 1
    return float(np.sum(dec.eigenvalues[start:end + 1]) / dec.total_variance)


# ---------------------------------------------------------------------------------------------
# MSSA (ssa_opt.h:3908-4283) and Cadzow (ssa_opt.h:3165-3290)
# ---------------------------------------------------------------------------------------------


def mssa_matvec(X: np.ndarray, v: np.ndarray, L: int) -> np.ndarray:
    """Stacked (M L) x K operator: y[m L + i] = sum_j X[m, i + j] v[j] (ssa_opt.h:4069-4083)."""
    return np.concatenate([hankel_matvec(X[m], v, L) for m in range(X.shape[0])], axis=0)


def mssa_matvec_T(X: np.ndarray, u: np.ndarray, L: int) -> np.ndarray:
    """z[j] = sum_m sum_i X[m, i + j] u[m L + i] (ssa_opt.h:4085-4101)."""
    M = X.shape[0]
    out = 0.0
    for m in range(M):
        out = out + hankel_matvec_T(X[m], u[m * L:(m + 1) * L], L)
    return out


def mssa_decompose(X: np.ndarray, L: int, k: int, oversampling: int, Omega: np.ndarray,
                   q: int = 0) -> Decomposition:
    """mssa_opt_decompose (ssa_opt.h:4116-4210) with a given Omega (K x kp); q as for SSA."""
    X = np.asarray(X, dtype=np.float64)
    Mch, N = X.shape
    K = N - L + 1
    ML = Mch * L
    p = 8 if oversampling <= 0 else oversampling
    kp = min(k + p, min(ML, K))
    k = min(k, kp)
    Om = np.asarray(Omega, dtype=np.float64)[:, :kp]
    Y = mssa_matvec(X, Om, L)
    Q, _ = np.linalg.qr(Y, mode="reduced")
    for _ in range(q):
        Z = mssa_matvec_T(X, Q, L)
        Qz, _ = np.linalg.qr(Z, mode="reduced")
        Y = mssa_matvec(X, Qz, L)
        Q, _ = np.linalg.qr(Y, mode="reduced")
    B = mssa_matvec_T(X, Q, L)
    B_left, S, B_right_T = np.linalg.svd(B, full_matrices=False)
    U = Q @ B_right_T.T[:, :k]
    V = B_left[:, :k].copy()
    sigma = S[:k].copy()
    _sign_fix(U, V)  # sum over all M L rows (:4195-4205)
    lam = sigma * sigma
    return Decomposition(U, V, sigma, lam, float(lam.sum()))


def mssa_reconstruct(dec: Decomposition, series_idx: int, group: Sequence[int], Mch: int, N: int,
                     L: int) -> np.ndarray:
    """mssa_opt_reconstruct (ssa_opt.h:4212-4242): per-channel block u_m = U[m L:(m+1) L]."""
    sub = Decomposition(dec.U[series_idx * L:(series_idx + 1) * L], dec.V, dec.sigma,
                        dec.eigenvalues, dec.total_variance)
    return reconstruct(sub, group, N, L)


def mssa_series_contributions(dec: Decomposition, Mch: int, L: int) -> np.ndarray:
    """contributions[m, i] = ||U[m L:(m+1) L, i]||^2 (ssa_opt.h:4255-4271), M x k."""
    k = dec.k
    out = np.zeros((Mch, k))
    for m in range(Mch):
        blk = dec.U[m * L:(m + 1) * L]
        out[m] = np.sum(blk * blk, axis=0)
    return out


def cadzow(x: np.ndarray, L: int, rank: int, max_iter: int, tol: float, Omega: np.ndarray,
           q: int = 0) -> tuple[np.ndarray, int, float, bool]:
    """ssa_opt_cadzow (ssa_opt.h:3165-3290) on the randomized branch (:3213-3217).

    Each iteration re-initialises a context, whose RNG restarts at the same seed (:1245), so
    every iteration uses the same Omega; it is passed in here. Returns
    (signal, iterations, final_diff, converged)."""
    y = np.asarray(x, dtype=np.float64).copy()
    N = len(y)
    K = N - L + 1
    ynorm = float(np.linalg.norm(y))
    if ynorm < 1e-15:
        ynorm = 1.0
    diff = 0.0
    converged = False
    it = 0
    group = list(range(rank))
    randomized = rank + 8 < min(L, K) // 2  # :3212
    while it < max_iter:
        if randomized:
            dec = decompose_randomized(y, L, rank, 8, Omega, q=q)
        else:  # :3227-3231, block size min(rank, 16), 3 iterations; Omega holds the start blocks
            dec = decompose_block(y, L, rank, min(rank, 16), 3, _split_blocks(Omega, rank, min(rank, 16)))
        y_new = reconstruct(dec, group, N, L)
        diff = float(np.linalg.norm(y_new - y)) / ynorm
        y = y_new
        it += 1
        if diff < tol:
            converged = True
            break
    return y, it, diff, converged


def _split_blocks(V0: np.ndarray, k: int, b: int) -> list:
    blocks, c = [], 0
    while c < k:
        cb = min(b, k - c)
        blocks.append(np.asarray(V0)[:, c:c + cb])
        c += cb
    return blocks


def cadzow_weighted(x: np.ndarray, L: int, rank: int, max_iter: int, tol: float, alpha: float,
                    Omega: np.ndarray, q: int = 0):
    """ssa_opt_cadzow_weighted (ssa_opt.h:3294-3315): alpha * cadzow(x) + (1 - alpha) * x."""
    y, it, diff, conv = cadzow(x, L, rank, max_iter, tol, Omega, q)
    if alpha < 1.0:
        y = alpha * y + (1.0 - alpha) * np.asarray(x, dtype=np.float64)
    return y, it, diff, conv


def cadzow_inplace(x: np.ndarray, L: int, rank: int, max_iter: int, tol: float,
                   omegas: Sequence[np.ndarray]):
    """ssa_opt_cadzow_inplace (ssa_opt.h:3319-3442) on a prepared context, randomized branch:
    iteration i draws the test matrix omegas[i]. The first reconstruction sets the norm; later
    ones are compared with the previous reconstruction; the signal is replaced by the
    reconstruction except after the last iteration. Returns (last reconstruction, iterations,
    final_diff, converged, signal held by the context)."""
    y = np.asarray(x, dtype=np.float64).copy()
    N = len(y)
    group = list(range(rank))
    y_norm, diff, converged = 1.0, 0.0, False
    y_prev = None
    y_new = None
    it = 0
    while it < max_iter:
        dec = decompose_randomized(y, L, rank, 8, omegas[it], q=0)
        y_new = reconstruct(dec, group, N, L)
        if it == 0:
            y_norm = float(np.linalg.norm(y_new))
            if y_norm < 1e-15:
                y_norm = 1.0
        else:
            diff = float(np.linalg.norm(y_new - y_prev)) / y_norm
            if diff < tol:
                converged = True
                it += 1
                break
        y_prev = y_new
        if it < max_iter - 1:
            y = y_new.copy()
        it += 1
    return y_new, it, diff, converged, y


def mssa_cadzow(X: np.ndarray, L: int, rank: int, iters: int, oversampling: int, omega: np.ndarray,
                q: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Multivariate Cadzow iterations on one instance X (M x N): each iteration projects the stacked
    (M L) x K trajectory operator of the current channels onto its leading `rank` components (the
    decomposition of mssa_decompose with the given K x kp start block `omega` and q subspace
    iterations, the same block every iteration, as the reference's fresh contexts restart their
    generator) and replaces every channel by its reconstruction (mssa_reconstruct of 0..rank-1),
    the reference's Cadzow loop (ssa_opt.h:3165-3290) applied to the multichannel operator
    (ssa_opt.h:3880-4283). Returns (channels, sigma of the last projection, relative change
    ||y_t - y_{t-1}|| / ||X|| per iteration)."""
    X = np.asarray(X, dtype=np.float64)
    Mch, N = X.shape
    xn = float(np.linalg.norm(X)) or 1.0
    y = X.copy()
    diffs = []
    d = None
    for _ in range(iters):
        d = mssa_decompose(y, L, rank, oversampling, omega, q=q)
        yn = np.stack([mssa_reconstruct(d, m, list(range(d.k)), Mch, N, L) for m in range(Mch)])
        diffs.append(float(np.linalg.norm(yn - y)) / xn)
        y = yn
    return y, d.sigma.copy(), np.array(diffs)


# ---------------------------------------------------------------------------------------------
# Synthetic workloads (seeded). Signals first, then Omega, from one numpy Generator (PCG64).
# ---------------------------------------------------------------------------------------------


def _noise_for_snr(rng: np.random.Generator, clean: np.ndarray, snr_db: float) -> np.ndarray:
    var = float(np.var(clean)) * 10.0 ** (-snr_db / 10.0)
    return rng.standard_normal(len(clean)) * math.sqrt(var)


def gaussian_omega(rng: np.random.Generator, K: int, kp: int) -> np.ndarray:
    """Omega ~ N(0,1), K x kp, drawn column by column (column-major as in ssa_opt.h:1719)."""
    return rng.standard_normal((kp, K)).T.copy()


def config1(seed: int = 0, N: int = 1000, L: int = 250, k: int = 50, p: int = 10):
    """Single series: x = 0.01 t + 2 sin(2 pi t/12) + sin(2 pi t/50 + phi) + noise at 7 dB."""
    rng = np.random.default_rng(seed)
    t = np.arange(N, dtype=np.float64)
    phi = rng.uniform(0.0, 2.0 * math.pi)
    clean = 0.01 * t + 2.0 * np.sin(2 * math.pi * t / 12) + np.sin(2 * math.pi * t / 50 + phi)
    x = clean + _noise_for_snr(rng, clean, 7.0)
    K = N - L + 1
    kp = min(k + p, L, K)
    Omega = gaussian_omega(rng, K, kp)
    return x, clean, Omega


def trend_two_sines(rng: np.random.Generator, N: int) -> tuple[np.ndarray, np.ndarray]:
    """Uniform-batch generator: linear trend + two sinusoids (periods U[6, 200], amplitudes
    U(0.5, 3)) + Gaussian noise at SNR U(0, 15) dB."""
    t = np.arange(N, dtype=np.float64)
    slope = rng.uniform(-0.002, 0.002)
    P = rng.uniform(6.0, 200.0, 2)
    A = rng.uniform(0.5, 3.0, 2)
    ph = rng.uniform(0.0, 2 * math.pi, 2)
    clean = slope * t + A[0] * np.sin(2 * math.pi * t / P[0] + ph[0]) + A[1] * np.sin(2 * math.pi * t / P[1] + ph[1])
    snr = rng.uniform(0.0, 15.0)
    return clean + _noise_for_snr(rng, clean, snr), clean


def config2_batch(B: int, seed: int = 1, N: int = 10000) -> np.ndarray:
    """B x N signals of the uniform batch (trend + two sinusoids + noise)."""
    rng = np.random.default_rng(seed)
    return np.stack([trend_two_sines(rng, N)[0] for _ in range(B)])


def walk_sines(rng: np.random.Generator, N: int) -> np.ndarray:
    """Uneven-batch generator: random-walk trend (sigma 0.05) + 1-3 sinusoids (periods
    U[4, N/10]) + Gaussian noise at SNR U(0, 15) dB."""
    t = np.arange(N, dtype=np.float64)
    clean = np.cumsum(rng.standard_normal(N) * 0.05)
    for _ in range(int(rng.integers(1, 4))):
        P = rng.uniform(4.0, max(5.0, N / 10.0))
        clean = clean + rng.uniform(0.5, 3.0) * np.sin(2 * math.pi * t / P + rng.uniform(0, 2 * math.pi))
    return clean + _noise_for_snr(rng, clean, rng.uniform(0.0, 15.0))


def config3_batch(B: int, seed: int = 2, nmin: int = 500, nmax: int = 20000):
    """Uneven batch: N log-uniform in [nmin, nmax], L = round(N/4), k uniform in {10..50}."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(B):
        N = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        L = max(2, int(round(N / 4)))
        k = int(rng.integers(10, 51))
        out.append((walk_sines(rng, N), L, k))
    return out


def config4_instance(rng: np.random.Generator, Mch: int = 16, N: int = 20000) -> np.ndarray:
    """MSSA instance: per-channel N(0,1) mixing of 4 shared sinusoids (periods U[10, 500]) +
    shared linear trend + independent noise at SNR 5 dB. Returns Mch x N."""
    t = np.arange(N, dtype=np.float64)
    P = rng.uniform(10.0, 500.0, 4)
    ph = rng.uniform(0.0, 2 * math.pi, 4)
    lat = np.stack([np.sin(2 * math.pi * t / P[j] + ph[j]) for j in range(4)])
    a = rng.uniform(-0.001, 0.001)
    X = np.zeros((Mch, N))
    for m in range(Mch):
        w = rng.standard_normal(4)
        clean = w @ lat + a * t
        X[m] = clean + _noise_for_snr(rng, clean, 5.0)
    return X


def reference_test_signal(N: int, seed: int = 42) -> np.ndarray:
    """generate_signal of MKL/test/ssa_opt_test.c:128-140 with its LCG + polar randn (:104-126)."""
    state = [seed & 0xFFFFFFFF]
    spare = [None]

    def lcg():
        state[0] = (state[0] * 1103515245 + 12345) & 0xFFFFFFFF
        return ((state[0] >> 16) & 0x7FFF) / 16384.0 - 1.0

    def randn():
        if spare[0] is not None:
            s = spare[0]
            spare[0] = None
            return s
        while True:
            u = lcg()
            v = lcg()
            s = u * u + v * v
            if 0 < s < 1:
                break
        s = math.sqrt(-2 * math.log(s) / s)
        spare[0] = v * s
        return u * s

    x = np.zeros(N)
    for i in range(N):
        t = i / N
        x[i] = 100.0 + 50.0 * t + 20.0 * math.sin(2 * math.pi * i / 100.0) + \
            10.0 * math.sin(2 * math.pi * i / 25.0) + 5.0 * randn()
    return x


# ---------------------------------------------------------------------------------------------
# Replica of the library's device Gaussian generator (checker side): the CUDA path draws
# Omega[row, col] for series s from SplitMix64 hashes of (seed_s, col, row // 2) followed by
# Box-Muller. The uniforms are bit-identical; the transform here is FP64 (the device uses FP32),
# so values agree to ~1e-7 relative.
# ---------------------------------------------------------------------------------------------

_M64 = (1 << 64) - 1


def _mix64(z):
    z = (z + 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def _mix64_np(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64)
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def series_seed(seed: int, s: int) -> int:
    """Seed of series s in a batch launched with `seed` (engine: seed ^ golden * (s + 1))."""
    return (seed ^ ((0x9E3779B97F4A7C15 * (s + 1)) & _M64)) & _M64


def single_series_seed(calls: int = 0) -> int:
    """Seed the single-series API uses for its `calls`-th generated test matrix (42 + 2^32 calls)."""
    return series_seed((42 + (calls << 32)) & _M64, 0)


def block_seed(calls: int = 0) -> int:
    """Seed of the single-series block method's `calls`-th start blocks; series 0's columns
    come from series_seed(block_seed(calls), 0), column c of the K x k start matrix being the
    generator's column c."""
    return ((42 + (calls << 32)) ^ 0xB10CB10CB10CB10C) & _M64


def mssa_seed(calls: int = 0) -> int:
    """Seed of an MSSA context's `calls`-th generated K x kp test matrix (used as is, with no
    per-series mixing: the channels share one matrix)."""
    return ((42 + (calls << 32)) ^ 0x4D55535341) & _M64


def device_gaussian(seed_s: int, K: int, kp: int) -> np.ndarray:
    """K x kp test matrix the device generates for a series with seed `seed_s`."""
    out = np.zeros((K, kp))
    npairs = (K + 1) // 2
    pairs = np.arange(npairs, dtype=np.uint64)
    for c in range(kp):
        key = _mix64((seed_s ^ ((0xD1B54A32D192ED03 * (c + 1)) & _M64)) & _M64)
        with np.errstate(over="ignore"):
            z = _mix64_np(np.uint64(key) + pairs)
        u1 = ((z >> np.uint64(40)).astype(np.float64) + 1.0) / 16777216.0
        u2 = ((z >> np.uint64(16)) & np.uint64(0xFFFFFF)).astype(np.float64) / 16777216.0
        r = np.sqrt(-2.0 * np.log(u1))
        vals = np.empty(2 * npairs)
        vals[0::2] = r * np.cos(2 * math.pi * u2)
        vals[1::2] = r * np.sin(2 * math.pi * u2)
        out[:, c] = vals[:K]
    return out
