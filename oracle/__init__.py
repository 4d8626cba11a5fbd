"""CPU oracle for the dense-factorization hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only as the checker or the timed CPU
reference; the CUDA library never routes through it.

Contents
--------
* ``potrf_residual`` / ``getrf_residual`` -- C restatement (``residual.c``) of
  the reference's CPU FP64 residual, ``include/utils/benchmark/cpu_fp64_residual.h:73-201``.
* ``potrf_residual_blas`` / ``getrf_residual_blas`` -- the same quantity with the
  FP64 product done by host BLAS (numpy), the analogue of the reference's
  ``HYGON_CPU_FP64_USE_CBLAS`` mode (``cpu_fp64_residual.h:52-71``); pinned
  against the C version on small sizes by the tests.
* ``potrf_residual_tiled`` / ``getrf_residual_tiled`` -- the same quantity block
  column by block column (host BLAS, a few FP64 blocks resident), for the
  orders 8192 ... 49152 of the sweep; pinned against the C version too.
* ``pivot_divergence`` -- first index where two pivot sequences differ and the
  FP64 relative gap of the two candidates there.
* ``pivot_agreement`` -- the same, plus the near-tie decision: the gap of the
  two candidates against the rounding error an FP32 factorization commits in
  them (unit roundoff x sqrt(j + 1) x (|a| + |L||U|) of the two rows).
* ``double_blocked_potrf`` / ``double_blocked_getrf`` -- plain-C FP32 restatement
  of the reference loops (``factor.c``).
* ``lapack_spotrf`` / ``lapack_sgetrf`` -- host LAPACK (SciPy's OpenBLAS), the
  pivot-sequence reference and the timed CPU baseline.
* ``uniform_pm1`` / ``spd_gram`` / ``general_uniform`` -- the seeded input
  generators (counter-based RNG, bit-identical to the device generator).
* ``scaled`` -- residual / (n * eps32), eps32 = 2**-23 (FLT_EPSILON).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
EPS32 = float(np.finfo(np.float32).eps)  # 2**-23
EPS64 = float(np.finfo(np.float64).eps)

_lib = None


def reference_root() -> str:
    """The reference checkout the oracle's _ref build reads (read-only):
    $HDBF_REFERENCE_ROOT, else /root/reference."""
    return os.environ.get("HDBF_REFERENCE_ROOT", "/root/reference")


def build() -> str:
    """Compile liboracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    ref = reference_root()
    if os.path.isdir(os.path.join(ref, "include")):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={ref}"], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        dp, ip, i = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int
        for name in ("oracle_potrf_residual_f32", "oracle_potrf_residual_f64"):
            f = getattr(L, name)
            f.restype = ctypes.c_double
            f.argtypes = [dp, dp, i, i, i, ip]
        for name in ("oracle_getrf_residual_f32", "oracle_getrf_residual_f64"):
            f = getattr(L, name)
            f.restype = ctypes.c_double
            f.argtypes = [dp, dp, dp, i, i, i, i, ip]
        L.oracle_double_blocked_potrf.restype = i
        L.oracle_double_blocked_potrf.argtypes = [dp, i, i, i, i, i]
        L.oracle_double_blocked_getrf.restype = i
        L.oracle_double_blocked_getrf.argtypes = [dp, i, i, i, i, dp]
        L.oracle_double_blocked_potrf_f64.restype = i
        L.oracle_double_blocked_potrf_f64.argtypes = [dp, i, i, i, i, i]
        L.oracle_double_blocked_getrf_f64.restype = i
        L.oracle_double_blocked_getrf_f64.argtypes = [dp, i, i, i, i, dp]
        for sfx in ("f32", "f64"):
            f = getattr(L, "oracle_recursive_potrf_" + sfx)
            f.restype = i
            f.argtypes = [dp, i, i, i]
            f = getattr(L, "oracle_blocked_right_looking_potrf_" + sfx)
            f.restype = i
            f.argtypes = [dp, i, i, i]
            f = getattr(L, "oracle_blocked_right_looking_getrf_" + sfx)
            f.restype = i
            f.argtypes = [dp, i, i, i, dp, i]
        for name in ("oracle_double_blocked_getrf_batched_f32",
                     "oracle_double_blocked_getrf_batched_f64"):
            f = getattr(L, name)
            f.restype = i
            f.argtypes = [dp, i, i, i, i, dp]
        L.oracle_parse_seed.restype = i
        L.oracle_parse_seed.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint)]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own residual header compiled in place (oracle/_ref)."""
    path = os.path.join(_HERE, "_ref", "libref_residual.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    dp, ip, i = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int
    for name in ("ref_potrf_residual_f32", "ref_potrf_residual_f64"):
        f = getattr(L, name)
        f.restype = ctypes.c_double
        f.argtypes = [dp, dp, i, i, i, ip]
    for name in ("ref_getrf_residual_f32", "ref_getrf_residual_f64"):
        f = getattr(L, name)
        f.restype = ctypes.c_double
        f.argtypes = [dp, dp, dp, i, i, i, i, ip]
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _colmajor(a, dtype):
    """Return (flat column-major buffer, lda) for a 2-D array or (flat, lda) tuple."""
    if isinstance(a, tuple):
        flat, lda = a
        return np.ascontiguousarray(flat, dtype=dtype).ravel(), int(lda)
    a = np.asarray(a, dtype=dtype)
    return np.asfortranarray(a).ravel(order="F"), a.shape[0]


def _call_residual(lib_, prefix, kind, factor, original, ipiv, n, lda, pivoting, tile):
    dt = factor.dtype
    suffix = "f64" if dt == np.float64 else "f32"
    err = ctypes.c_int(0)
    if kind == "potrf":
        f = getattr(lib_, f"{prefix}_potrf_residual_{suffix}")
        r = f(_ptr(factor), _ptr(original), n, lda, tile, ctypes.byref(err))
    else:
        piv = None if ipiv is None else np.ascontiguousarray(ipiv, dtype=np.int32)
        f = getattr(lib_, f"{prefix}_getrf_residual_{suffix}")
        r = f(_ptr(factor), _ptr(original), _ptr(piv), n, lda, int(pivoting), tile,
              ctypes.byref(err))
    if err.value:
        raise ValueError("invalid residual inputs")
    return float(r)


def potrf_residual(L, A, n, lda, tile=512, impl="oracle"):
    """||A - L L^T||_F / ||A||_F in FP64 (flat column-major buffers with lda)."""
    L = np.ascontiguousarray(L)
    A = np.ascontiguousarray(A, dtype=L.dtype)
    lib_ = lib() if impl == "oracle" else ref_lib()
    return _call_residual(lib_, "oracle" if impl == "oracle" else "ref", "potrf",
                          L, A, None, n, lda, False, tile)


def getrf_residual(LU, A, ipiv, n, lda, pivoting=True, tile=512, impl="oracle"):
    """||P A - L U||_F / ||A||_F in FP64; ipiv 1-based global LAPACK pivots."""
    LU = np.ascontiguousarray(LU)
    A = np.ascontiguousarray(A, dtype=LU.dtype)
    lib_ = lib() if impl == "oracle" else ref_lib()
    return _call_residual(lib_, "oracle" if impl == "oracle" else "ref", "getrf",
                          LU, A, ipiv, n, lda, pivoting, tile)


def scaled(residual: float, n: int) -> float:
    """Residual scaled by n * eps32 (eps32 = 2**-23)."""
    return residual / (n * EPS32)


# --- BLAS-backed residuals (same definition, FP64 product by host BLAS) -----

def _ssq_norm(x: np.ndarray) -> float:
    if not np.all(np.isfinite(x)):
        return float("inf")
    s = np.max(np.abs(x)) if x.size else 0.0
    if s == 0.0:
        return 0.0
    return float(s * np.sqrt(np.sum((x / s) ** 2)))


def _ratio(num: float, den: float) -> float:
    if not np.isfinite(num) or not np.isfinite(den):
        return float("inf")
    if den == 0.0:
        return 0.0 if num == 0.0 else float("inf")
    return num / den


def potrf_residual_blas(L2d: np.ndarray, A2d: np.ndarray) -> float:
    """2-D n x n arrays; uses the lower triangle of L2d."""
    L = np.tril(np.asarray(L2d, dtype=np.float64))
    A = np.asarray(A2d, dtype=np.float64)
    R = L @ L.T - A
    return _ratio(_ssq_norm(R), _ssq_norm(A))


def ipiv_to_perm(ipiv, n):
    perm = np.arange(n)
    for r in range(n):
        p = int(ipiv[r]) - 1
        if p < r or p >= n:
            return None
        perm[r], perm[p] = perm[p], perm[r]
    return perm


def getrf_residual_blas(LU2d: np.ndarray, A2d: np.ndarray, ipiv) -> float:
    n = LU2d.shape[0]
    perm = ipiv_to_perm(ipiv, n)
    if perm is None:
        return float("inf")
    LU = np.asarray(LU2d, dtype=np.float64)
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    PA = np.asarray(A2d, dtype=np.float64)[perm, :]
    return _ratio(_ssq_norm(L @ U - PA), _ssq_norm(PA))


# --- tiled BLAS residuals for large orders ---------------------------------
#
# The same quantities as potrf_residual / getrf_residual
# (cpu_fp64_residual.h:73-201: FP32 values widened to FP64 before they are
# multiplied, structurally zero triangular products skipped, Frobenius norms
# of the whole residual and of the whole original), computed block column by
# block column with host BLAS so that orders of 32768 and 49152 finish in
# seconds to minutes on the host's cores and hold only a few column blocks in
# FP64 at a time.  The norms merge per-block (scale, sum of squares) pairs as
# the reference's overflow-safe accumulation does (cpu_fp64_residual.h:29-50).

class _Ssq:
    def __init__(self):
        self.scale, self.sumsq, self.finite = 0.0, 1.0, True

    def add(self, x: np.ndarray):
        if x.size == 0:
            return
        hi, lo = float(np.max(x)), float(np.min(x))
        m = max(abs(hi), abs(lo))
        if not np.isfinite(m) or np.isnan(hi) or np.isnan(lo):
            self.finite = False
            return
        if m == 0.0:
            return
        if 1e-150 < m < 1e150:  # no overflow or underflow of x*x: plain dot
            flat = np.ascontiguousarray(x).ravel(order="K")
            s = float(np.dot(flat, flat)) / (m * m)
        else:
            s = float(np.sum(np.square(x / m)))
        if self.scale < m:
            self.sumsq = s + self.sumsq * (self.scale / m) ** 2
            self.scale = m
        else:
            self.sumsq += s * (m / self.scale) ** 2

    def norm(self) -> float:
        if not self.finite:
            return float("inf")
        return self.scale * float(np.sqrt(self.sumsq)) if self.scale > 0 else 0.0


def _ssq_ratio(num: _Ssq, den: _Ssq) -> float:
    if not num.finite or not den.finite:
        return float("inf")
    if den.scale == 0.0:
        return 0.0 if num.scale == 0.0 else float("inf")
    return (num.scale / den.scale) * float(np.sqrt(num.sumsq / den.sumsq))


def potrf_residual_tiled(L2d: np.ndarray, A2d: np.ndarray, block: int = 4096) -> float:
    """||A - L L^T||_F / ||A||_F in FP64 for n x n arrays (L2d: lower factor;
    its strict upper triangle is ignored).  One lower block column of L L^T
    is formed per step; each computed product entry (r, c), r >= c, is compared
    with A(r, c) and, for r > c outside the diagonal block, with A(c, r)."""
    n = A2d.shape[0]
    num, den = _Ssq(), _Ssq()
    for j0 in range(0, n, block):
        j1 = min(n, j0 + block)
        X = np.array(L2d[j0:, :j1], dtype=np.float64, order="F")  # rows j0..n, columns 0..j1
        for c in range(j1 - j0):  # diagonal block: lower triangle only
            X[:c, j0 + c] = 0.0
        P = X @ X[: j1 - j0, :].T                           # (L L^T)[j0:n, j0:j1]
        del X
        D = P[: j1 - j0] - A2d[j0:j1, j0:j1]
        num.add(D)
        den.add(np.asarray(A2d[j0:j1, j0:j1], dtype=np.float64))
        if j1 < n:
            low = np.asarray(A2d[j1:, j0:j1], dtype=np.float64)
            up = np.asarray(A2d[j0:j1, j1:], dtype=np.float64)
            num.add(P[j1 - j0:] - low)
            num.add(P[j1 - j0:].T - up)
            den.add(low)
            den.add(up)
        del P
    return _ssq_ratio(num, den)


def getrf_residual_tiled(LU2d: np.ndarray, A2d: np.ndarray, ipiv, block: int = 4096) -> float:
    """||P A - L U||_F / ||A||_F in FP64 for n x n arrays; ipiv 1-based LAPACK
    pivots (an invalid pivot gives +inf, cpu_fp64_residual.h:157-163).  One
    block column of L U is formed per step from the trapezoidal blocks of L
    that can reach it."""
    n = A2d.shape[0]
    perm = ipiv_to_perm(ipiv, n)
    if perm is None:
        return float("inf")
    num, den = _Ssq(), _Ssq()
    for j0 in range(0, n, block):
        j1 = min(n, j0 + block)
        P = np.zeros((n, j1 - j0), dtype=np.float64)
        for k0 in range(0, j1, block):
            k1 = min(n, k0 + block)
            Lk = np.array(LU2d[k0:, k0:k1], dtype=np.float64, order="F")  # rows k0..n
            for c in range(k1 - k0):  # unit lower diagonal block
                Lk[:c, c] = 0.0
                Lk[c, c] = 1.0
            Uk = np.array(LU2d[k0:k1, j0:j1], dtype=np.float64, order="F")
            if k0 == j0:
                for c in range(j1 - j0):  # upper diagonal block
                    Uk[c + 1:, c] = 0.0
            P[k0:] += Lk @ Uk
            del Lk
        PA = np.asarray(np.asarray(A2d[:, j0:j1])[perm], dtype=np.float64)
        num.add(P - PA)
        den.add(PA)
        del P, PA
    return _ssq_ratio(num, den)


# --- reference loops restated in C (FP32 and FP64) -------------------------

def double_blocked_potrf(A2d: np.ndarray, nb: int, b: int, syrk_k_tile: int = 0):
    A = np.asfortranarray(np.array(A2d, dtype=np.float32))
    n = A.shape[0]
    info = lib().oracle_double_blocked_potrf(A.ctypes.data_as(ctypes.c_void_p), n, n,
                                             nb, b, syrk_k_tile)
    return A, info


def double_blocked_potrf_f64(A2d: np.ndarray, nb: int, b: int, syrk_k_tile: int = 0):
    """FP64 twin of double_blocked_potrf (the same loops in double)."""
    A = np.asfortranarray(np.array(A2d, dtype=np.float64))
    n = A.shape[0]
    info = lib().oracle_double_blocked_potrf_f64(A.ctypes.data_as(ctypes.c_void_p), n, n,
                                                 nb, b, syrk_k_tile)
    return A, info


def double_blocked_getrf_f64(A2d: np.ndarray, outer_nb: int, inner_nb: int):
    """FP64 twin of double_blocked_getrf (the same loops in double)."""
    A = np.asfortranarray(np.array(A2d, dtype=np.float64))
    n = A.shape[0]
    ipiv = np.zeros(n, dtype=np.int32)
    info = lib().oracle_double_blocked_getrf_f64(A.ctypes.data_as(ctypes.c_void_p), n, n,
                                                 outer_nb, inner_nb,
                                                 ipiv.ctypes.data_as(ctypes.c_void_p))
    return A, ipiv, info


def double_blocked_getrf_batched(A2d: np.ndarray, outer_nb: int, inner_nb: int,
                                 dtype=np.float32):
    """Batched-pivot schedule of the double-blocked LU (FP32 or FP64)."""
    A = np.asfortranarray(np.array(A2d, dtype=dtype))
    n = A.shape[0]
    ipiv = np.zeros(n, dtype=np.int32)
    fn = (lib().oracle_double_blocked_getrf_batched_f64 if A.dtype == np.float64
          else lib().oracle_double_blocked_getrf_batched_f32)
    info = fn(A.ctypes.data_as(ctypes.c_void_p), n, n, outer_nb, inner_nb,
              ipiv.ctypes.data_as(ctypes.c_void_p))
    return A, ipiv, info


def recursive_potrf(A2d: np.ndarray, nb: int, dtype=np.float32):
    """Recursive Cholesky (FP32 or FP64)."""
    A = np.asfortranarray(np.array(A2d, dtype=dtype))
    n = A.shape[0]
    sfx = "f64" if A.dtype == np.float64 else "f32"
    info = getattr(lib(), "oracle_recursive_potrf_" + sfx)(
        A.ctypes.data_as(ctypes.c_void_p), n, n, nb)
    return A, info


def blocked_right_looking_potrf(A2d: np.ndarray, nb: int, dtype=np.float32):
    """Right-looking blocked Cholesky (FP32 or FP64)."""
    A = np.asfortranarray(np.array(A2d, dtype=dtype))
    n = A.shape[0]
    sfx = "f64" if A.dtype == np.float64 else "f32"
    info = getattr(lib(), "oracle_blocked_right_looking_potrf_" + sfx)(
        A.ctypes.data_as(ctypes.c_void_p), n, n, nb)
    return A, info


def blocked_right_looking_getrf(A2d: np.ndarray, nb: int, pivot: bool = True,
                                dtype=np.float32):
    """Right-looking blocked LU, pivoted or NPVT (FP32 or FP64)."""
    A = np.asfortranarray(np.array(A2d, dtype=dtype))
    n = A.shape[0]
    ipiv = np.zeros(max(n, 1), dtype=np.int32)
    sfx = "f64" if A.dtype == np.float64 else "f32"
    info = getattr(lib(), "oracle_blocked_right_looking_getrf_" + sfx)(
        A.ctypes.data_as(ctypes.c_void_p), n, n, nb, ipiv.ctypes.data_as(ctypes.c_void_p),
        1 if pivot else 0)
    return A, ipiv[:n], info


def double_blocked_getrf(A2d: np.ndarray, outer_nb: int, inner_nb: int):
    A = np.asfortranarray(np.array(A2d, dtype=np.float32))
    n = A.shape[0]
    ipiv = np.zeros(n, dtype=np.int32)
    info = lib().oracle_double_blocked_getrf(A.ctypes.data_as(ctypes.c_void_p), n, n,
                                             outer_nb, inner_nb,
                                             ipiv.ctypes.data_as(ctypes.c_void_p))
    return A, ipiv, info


def pivot_divergence(A2d: np.ndarray, ipiv_a, ipiv_b):
    """First index where two LAPACK pivot sequences differ, and how close the
    pivot choice was there.

    Returns (None, None) when identical.  Otherwise (j, rel_gap): the common
    prefix of pivots is applied to A, the Schur complement column j is formed
    in FP64 (S = A22 - A21 A11^{-1} A12, column j), and rel_gap = (|s|_1st -
    |s|_2nd) / |s|_1st over the candidate rows.  A rel_gap at the level of FP32
    rounding (<~ 1e-4) marks a near-tie, where any FP32 implementation may
    legitimately choose either row.
    """
    a = np.asarray(ipiv_a).astype(np.int64)
    b = np.asarray(ipiv_b).astype(np.int64)
    diff = np.nonzero(a != b)[0]
    if diff.size == 0:
        return None, None
    j = int(diff[0])
    n = A2d.shape[0]
    perm = np.arange(n)
    for r in range(j):
        p = a[r] - 1
        perm[r], perm[p] = perm[p], perm[r]
    M = np.asarray(A2d[:, : j + 1], dtype=np.float64)[perm, :]  # only columns 0..j matter
    if j > 0:
        x = np.linalg.solve(M[:j, :j], M[:j, j])
        col = M[j:, j] - M[j:, :j] @ x
    else:
        col = M[:, 0].copy()
    mag = np.sort(np.abs(col))[::-1]
    gap = (mag[0] - mag[1]) / mag[0] if mag.size > 1 and mag[0] > 0 else 0.0
    return j, float(gap)


NEAR_TIE = 1e-4
# A divergence is a near-tie when the two candidates' exact Schur-complement
# magnitudes differ by less than TIE_ROUNDING times the typical rounding error
# of a computed entry, u sqrt(j + 1) (|a_ij| + sum_k |l_ik| |u_kj|) (the
# rounding-error bound of LU with the square-root growth of random rounding
# errors in place of the worst-case j u).  Two FP32 implementations that sum
# in different orders both commit that much, so either row is a correct
# partial-pivoting choice within FP32 arithmetic.
TIE_ROUNDING = 2.0


def _lu_nopivot(M: np.ndarray) -> np.ndarray:
    """In-place FP64 LU without pivoting of a square matrix whose rows are
    already in pivot order (blocked right-looking, host BLAS)."""
    from scipy.linalg import solve_triangular
    n = M.shape[0]
    nb = 128
    for k in range(0, n, nb):
        e = min(k + nb, n)
        for c in range(k, e):
            M[c + 1:, c] /= M[c, c]
            M[c + 1:, c + 1:e] -= np.outer(M[c + 1:, c], M[c, c + 1:e])
        if e < n:
            M[k:e, e:] = solve_triangular(M[k:e, k:e], M[k:e, e:], lower=True,
                                          unit_diagonal=True, check_finite=False)
            M[e:, e:] -= M[e:, k:e] @ M[k:e, e:]
    return M


def pivot_agreement(A2d: np.ndarray, ipiv_ref, ipiv, unit_roundoff: float = 2.0 ** -24,
                    rel_tie: float = NEAR_TIE) -> dict:
    """Compare a pivot sequence with a reference one (both LAPACK 1-based).

    Returns {"first_divergence": None} when identical; otherwise the first
    differing column j, the FP64 relative gap of the two largest candidates
    of the exact Schur complement column j (common pivot prefix applied),
    "gap_over_rounding" = their absolute gap / (u sqrt(j + 1) s), s the larger
    of |a_ij| + sum_k |l_ik| |u_kj| over the two rows (FP64 LU without
    pivoting of the permuted leading block), and "near_tie": rel_gap < rel_tie
    or gap_over_rounding <= TIE_ROUNDING.
    """
    from scipy.linalg import solve_triangular
    a = np.asarray(ipiv_ref).astype(np.int64)
    b = np.asarray(ipiv).astype(np.int64)
    diff = np.nonzero(a != b)[0]
    if diff.size == 0:
        return {"first_divergence": None, "near_tie": True}
    j = int(diff[0])
    n = A2d.shape[0]
    perm = np.arange(n)
    for r in range(j):
        p = a[r] - 1
        perm[r], perm[p] = perm[p], perm[r]
    M = np.asarray(A2d[:, : j + 1], dtype=np.float64)[perm, :]
    if j > 0:
        LU11 = _lu_nopivot(M[:j, :j].copy())
        u12 = solve_triangular(LU11, M[:j, j], lower=True, unit_diagonal=True,
                               check_finite=False)
        x = solve_triangular(LU11, u12, lower=False, check_finite=False)
        col = M[j:, j] - M[j:, :j] @ x  # Schur complement column j

        def scale_of(i):  # |a_ij| + |l_i||u_j|, l_i = M[i, :j] U11^{-1}
            li = solve_triangular(LU11, M[j + i, :j], trans="T", lower=False,
                                  check_finite=False)
            return float(abs(M[j + i, j]) + np.abs(li) @ np.abs(u12))
    else:
        col = M[:, 0].copy()

        def scale_of(i):
            return float(abs(col[i]))
    order = np.argsort(-np.abs(col), kind="stable")
    mag = np.abs(col)[order]
    if mag.size < 2 or mag[0] == 0:
        return {"first_divergence": j, "rel_gap": 0.0, "gap_over_rounding": 0.0,
                "near_tie": True}
    gap = float(mag[0] - mag[1])
    rel = gap / float(mag[0])
    s = max(scale_of(int(order[0])), scale_of(int(order[1])))
    tau = unit_roundoff * np.sqrt(j + 1.0) * s
    ratio = gap / tau if tau > 0 else float("inf")
    return {"first_divergence": j, "rel_gap": rel, "gap_over_rounding": float(ratio),
            "near_tie": bool(rel < rel_tie or ratio <= TIE_ROUNDING)}


def parse_seed(text):
    seed = ctypes.c_uint(19)
    ok = lib().oracle_parse_seed(None if text is None else text.encode(), ctypes.byref(seed))
    return bool(ok), seed.value


# --- host LAPACK (SciPy OpenBLAS) -------------------------------------------

def lapack_spotrf(A2d: np.ndarray):
    from scipy.linalg import lapack
    c, info = lapack.spotrf(np.asfortranarray(A2d, dtype=np.float32), lower=1,
                            clean=0, overwrite_a=0)
    return c, int(info)


def lapack_sgetrf(A2d: np.ndarray):
    """Returns (packed LU, 1-based ipiv, info) like LAPACK sgetrf."""
    from scipy.linalg import lapack
    lu, piv, info = lapack.sgetrf(np.asfortranarray(A2d, dtype=np.float32), overwrite_a=0)
    return lu, (piv + 1).astype(np.int32), int(info)


def lapack_dgetrf(A2d: np.ndarray):
    from scipy.linalg import lapack
    lu, piv, info = lapack.dgetrf(np.asfortranarray(A2d, dtype=np.float64), overwrite_a=0)
    return lu, (piv + 1).astype(np.int32), int(info)


# --- seeded generators (bit-identical to the device generator) --------------

_M64 = (1 << 64) - 1
_GOLD = np.uint64(0x9E3779B97F4A7C15)
_MIX = np.uint64(0xD1B54A32D192ED03)


def _splitmix(x: np.ndarray) -> np.ndarray:
    x = x ^ (x >> np.uint64(30))
    x = x * np.uint64(0xBF58476D1CE4E5B9)
    x = x ^ (x >> np.uint64(27))
    x = x * np.uint64(0x94D049BB133111EB)
    x = x ^ (x >> np.uint64(31))
    return x


def uniform_pm1(count: int, seed: int, offset: int = 0) -> np.ndarray:
    """Counter-based U[-1,1) FP32: element i = top-24-bit(h(seed, i)) / 2**23 - 1.

    h(seed, i) = splitmix64_finalize(seed * 0x9E3779B97F4A7C15 + (i + 1) * 0xD1B54A32D192ED03)
    (all mod 2**64).  Every value is a multiple of 2**-23 in [-1, 1), so it is
    exact in FP32 and identical on host and device.
    """
    with np.errstate(over="ignore"):
        idx = np.arange(offset, offset + count, dtype=np.uint64) + np.uint64(1)
        x = np.uint64(seed) * _GOLD + idx * _MIX
        x = _splitmix(x)
    top = (x >> np.uint64(40)).astype(np.float64)
    return (top / float(1 << 23) - 1.0).astype(np.float32)


def general_uniform(n: int, seed: int) -> np.ndarray:
    """n x n FP32 with iid U[-1,1) entries (column-major linear index)."""
    return uniform_pm1(n * n, seed).reshape(n, n, order="F")


def orthogonal(n: int, seed: int) -> np.ndarray:
    """Q from the QR factorization of an iid N(0,1) matrix (sign-fixed)."""
    rng = np.random.default_rng(seed)
    Q, R = np.linalg.qr(rng.standard_normal((n, n)))
    return Q * np.sign(np.diag(R))


def spd_kappa(n: int, kappa: float, seed: int) -> np.ndarray:
    """FP64 SPD A = Q diag(lambda) Q^T, lambda log-spaced in [1, kappa]."""
    Q = orthogonal(n, seed)
    lam = np.logspace(0.0, np.log10(kappa), n)
    A = (Q * lam) @ Q.T
    return 0.5 * (A + A.T)


def general_kappa(n: int, kappa: float, seed: int) -> np.ndarray:
    """FP64 general A = U diag(sigma) V^T, sigma log-spaced in [1, kappa]."""
    U = orthogonal(n, seed)
    V = orthogonal(n, seed + 7919)
    sig = np.logspace(0.0, np.log10(kappa), n)
    return (U * sig) @ V.T


def backward_error(A: np.ndarray, X: np.ndarray, B: np.ndarray) -> float:
    """max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf) in FP64."""
    R = B - A @ X
    an = np.abs(A).sum(axis=1).max()
    num = np.abs(R).max(axis=0)
    den = an * np.abs(X).max(axis=0) + np.abs(B).max(axis=0)
    return float((num / den).max())


def spd_gram(n: int, seed: int) -> np.ndarray:
    """A = G G^T / n + I formed in FP64 then rounded to FP32 (G iid U[-1,1) FP32)."""
    G = general_uniform(n, seed).astype(np.float64)
    A = (G @ G.T) / n + np.eye(n)
    A = 0.5 * (A + A.T)
    return A.astype(np.float32)
