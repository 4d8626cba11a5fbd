"""GPU tests of the building-block entry points (GEMM / SYRK / TRSM / aux)
against FP64 references of the same operation (tolerances stated per test)."""
import numpy as np
import pytest

import oracle
from tests.common import dev, host2d, ptr

pytestmark = pytest.mark.gpu


def rnd(shape, seed):
    return np.random.default_rng(seed).uniform(-1, 1, size=shape).astype(np.float32)


def put(torch, M, ld, fill=np.nan):
    buf = np.full((ld, M.shape[1]), fill, dtype=np.float32)
    buf[: M.shape[0]] = M
    return dev(torch, buf)


def rel_err(got, want):
    return np.abs(got.astype(np.float64) - want).max() / max(1e-30, np.abs(want).max())


# FP32 accumulation over k terms of magnitude <= 1: |err| <~ k * eps32 * max|terms|
def tol(k):
    return 4 * max(k, 16) * 2.0 ** -23


@pytest.mark.parametrize("M,N,K,pad", [(1, 1, 1, 0), (5, 7, 3, 1), (128, 128, 8, 0), (129, 131, 17, 2),
                                       (300, 64, 257, 0), (1000, 600, 300, 3), (4096, 256, 1024, 0)])
def test_gemm_nt_update(hd, handle, torch_cuda, M, N, K, pad):
    A, B, C = rnd((M, K), 1), rnd((N, K), 2), rnd((M, N), 3)
    lda, ldb, ldc = M + pad, N + pad, M + pad
    dA, dB, dC = put(torch_cuda, A, lda), put(torch_cuda, B, ldb), put(torch_cuda, C, ldc)
    hd.call("gemm_nt_update", handle.ptr, M, N, K, ptr(dA), lda, ptr(dB), ldb, ptr(dC), ldc)
    torch_cuda.cuda.synchronize()
    handle.check()
    got = host2d(dC, ldc, ldc, N)
    want = C.astype(np.float64) - A.astype(np.float64) @ B.astype(np.float64).T
    assert rel_err(got[:M], want) <= tol(K)
    if pad:
        assert np.all(np.isnan(got[M:]))


@pytest.mark.parametrize("M,N,K", [(256, 1, 1), (300, 8, 33), (4096, 16, 1024), (5000, 31, 4099),
                                   (70000, 32, 96), (1024, 9, 20000)])
def test_gemm_nt_update_skinny(hd, handle, torch_cuda, M, N, K):
    # narrow updates take the row-per-thread kernel; with the workspace
    # reserved, long K is split across CTAs and reduced in a fixed order
    handle.reserve(256 << 20)
    A, B, C = rnd((M, K), 11), rnd((N, K), 12), rnd((M, N), 13)
    lda, ldb, ldc = M + 3, N + 1, M + 5
    dA, dB, dC = put(torch_cuda, A, lda), put(torch_cuda, B, ldb), put(torch_cuda, C, ldc)
    hd.call("gemm_nt_update", handle.ptr, M, N, K, ptr(dA), lda, ptr(dB), ldb, ptr(dC), ldc)
    torch_cuda.cuda.synchronize()
    handle.check()
    got = host2d(dC, ldc, ldc, N)
    want = C.astype(np.float64) - A.astype(np.float64) @ B.astype(np.float64).T
    assert rel_err(got[:M], want) <= tol(K)
    assert np.all(np.isnan(got[M:]))


def test_gemm_nt_update_m_tiled(hd, handle, torch_cuda):
    M, N, K = 1000, 200, 96
    A, B, C = rnd((M, K), 4), rnd((N, K), 5), rnd((M, N), 6)
    dA, dB, dC = dev(torch_cuda, A), dev(torch_cuda, B), dev(torch_cuda, C)
    hd.call("gemm_nt_update_m_tiled", handle.ptr, M, N, K, ptr(dA), M, ptr(dB), N, ptr(dC), M, 333)
    torch_cuda.cuda.synchronize()
    want = C.astype(np.float64) - A.astype(np.float64) @ B.astype(np.float64).T
    assert rel_err(host2d(dC, M, M, N), want) <= tol(K)


@pytest.mark.parametrize("n,k,tk", [(1, 1, 0), (130, 70, 0), (513, 300, 128), (1024, 2048, 1000)])
def test_syrk_lower_kblocked(hd, handle, torch_cuda, n, k, tk):
    A, C = rnd((n, k), 7), rnd((n, n), 8)
    dA, dC = dev(torch_cuda, A), dev(torch_cuda, C)
    hd.call("syrk_lower_update_kblocked", handle.ptr, n, k, ptr(dA), n, ptr(dC), n, tk)
    torch_cuda.cuda.synchronize()
    handle.check()
    got = host2d(dC, n, n, n)
    want = C.astype(np.float64) - A.astype(np.float64) @ A.astype(np.float64).T
    lo = np.tril_indices(n)
    assert rel_err(got[lo], want[lo]) <= tol(k)
    up = np.triu_indices(n, 1)
    np.testing.assert_array_equal(got[up], C[up])


@pytest.mark.parametrize("fn", ["recursive_syrk_parallel", "batched_syrk_bottom_up"])
def test_recursive_and_batched_syrk(hd, handle, torch_cuda, fn):
    n, k, nb = 700, 160, 128
    A, C = rnd((n, k), 9), rnd((n, n), 10)
    dA, dC = dev(torch_cuda, A), dev(torch_cuda, C)
    if fn == "recursive_syrk_parallel":
        hd.call(fn, handle.ptr, ptr(dA), n, ptr(dC), n, n, k, nb)
    else:
        hd.call(fn, handle.ptr, None, ptr(dA), n, ptr(dC), n, n, k, nb)
    torch_cuda.cuda.synchronize()
    handle.check()
    got = host2d(dC, n, n, n)
    want = C.astype(np.float64) - A.astype(np.float64) @ A.astype(np.float64).T
    lo = np.tril_indices(n)
    assert rel_err(got[lo], want[lo]) <= tol(k)


def lower_factor(m, seed):
    L = np.tril(rnd((m, m), seed)) * 0.1
    L[np.diag_indices(m)] = 1.0 + np.abs(rnd((m,), seed + 1))
    return L.astype(np.float32)


@pytest.mark.parametrize("fn,extra", [("trsm_right_lower_transpose", ()),
                                      ("double_blocked_trsm", (256, 96)),
                                      ("recursive_trsm", (64,)),
                                      ("recursive_trsm_tiled_update", (100,)),
                                      ("iterative_trsm_right_looking", (70,))])
@pytest.mark.parametrize("rows,m", [(1, 1), (33, 65), (1000, 300)])
def test_right_trsm_family(hd, handle, torch_cuda, fn, extra, rows, m):
    L = lower_factor(m, 11)
    B = rnd((rows, m), 12)
    dL, dB = dev(torch_cuda, L), dev(torch_cuda, B)
    if fn == "trsm_right_lower_transpose":
        hd.call(fn, handle.ptr, rows, m, ptr(dL), m, ptr(dB), rows)
    elif fn == "double_blocked_trsm":
        hd.call(fn, handle.ptr, ptr(dL), m, ptr(dB), rows, rows, m, *extra)
    else:
        hd.call(fn, handle.ptr, ptr(dL), m, ptr(dB), rows, rows, m, *extra)
    torch_cuda.cuda.synchronize()
    handle.check()
    want = np.linalg.solve(L.astype(np.float64), B.astype(np.float64).T).T  # X L^T = B
    got = host2d(dB, rows, rows, m)
    assert rel_err(got, want) <= 1e-4


def test_add_damping_and_auto_scale(hd, handle, torch_cuda):
    n = 200
    A = oracle.spd_gram(n, 1) * np.float32(3)
    dA = dev(torch_cuda, A)
    stream = torch_cuda.cuda.current_stream().cuda_stream
    hd.call("launch_add_damping", ptr(dA), n, n, np.float32(0.5), stream)
    torch_cuda.cuda.synchronize()
    got = host2d(dA, n, n, n)
    want = A.copy()
    want[np.diag_indices(n)] += np.float32(0.5)
    np.testing.assert_array_equal(got, want)
    mx = torch_cuda.zeros(1, dtype=torch_cuda.int32, device="cuda")
    hd.call("launch_auto_scale", ptr(dA), n, n, ptr(mx), False, stream)
    torch_cuda.cuda.synchronize()
    s = host2d(dA, n, n, n)
    f = np.float32(65504.0) / np.abs(np.diag(want)).max()
    lo = np.tril_indices(n)
    np.testing.assert_allclose(s[lo], want[lo] * f, rtol=1e-6)
    np.testing.assert_array_equal(s[np.triu_indices(n, 1)], want[np.triu_indices(n, 1)])


def test_fp16_round_trip(hd, handle, torch_cuda):
    rows, cols = 77, 13
    X = rnd((rows, cols), 3) * np.float32(100)
    dX = dev(torch_cuda, X)
    h = torch_cuda.zeros(80 * cols, dtype=torch_cuda.float16, device="cuda")
    y = torch_cuda.zeros(90 * cols, dtype=torch_cuda.float32, device="cuda")
    stream = torch_cuda.cuda.current_stream().cuda_stream
    hd.call("launch_fp32_to_fp16", ptr(dX), ptr(h), rows, cols, rows, 80, stream)
    hd.call("launch_fp16_to_fp32", ptr(h), ptr(y), rows, cols, 80, 90, stream)
    torch_cuda.cuda.synchronize()
    got = host2d(y, 90, 90, cols)[:rows]
    np.testing.assert_array_equal(got, X.astype(np.float16).astype(np.float32))
