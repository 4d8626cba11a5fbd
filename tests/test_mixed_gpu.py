"""GPU tests of the mixed-precision factorizations (tcgen05 trailing updates),
the FP32 solves, and FP64 iterative refinement, all through the C ABI.

Bounds: a factorization whose trailing updates round their operands to a
16-bit format with unit roundoff u has a backward error of order u, so the
unscaled CPU FP64 residual ||A - LL^T||/||A|| (||PA - LU||/||A||) is checked
against 8u (one product) or 8u^2-level split modes (tol stated per test).
Refinement must reach the FP64 normwise backward error tolerance 1e-13."""
import ctypes

import numpy as np
import pytest

import hygondoubleblockedfactorizations_b200 as hd_mod
import oracle
from tests.common import dev, host2d, info_tensor, padded, ptr

pytestmark = pytest.mark.gpu

U = {"bf16": 2.0 ** -8, "fp16": 2.0 ** -11, "bf16x3": 2.0 ** -16, "fp16x3": 2.0 ** -21}


def potrf_resid(L, A):
    return oracle.potrf_residual_blas(np.tril(L), A)


@pytest.mark.parametrize("prec", ["bf16", "fp16", "bf16x3", "fp16x3"])
@pytest.mark.parametrize("n,nb", [(1000, 256), (1536, 512)])
def test_spotrf_mixed(hd, handle, torch_cuda, prec, n, nb):
    A = oracle.spd_gram(n, 0)
    dA = dev(torch_cuda, A)
    info = info_tensor(torch_cuda)
    st = hd.call("hdbf_spotrf_mixed", handle.ptr, hd_mod.PREC[prec], ptr(dA), n, n, nb, ptr(info))
    torch_cuda.cuda.synchronize()
    assert st == 0 and int(info.item()) == 0
    assert handle.device_errors() == 0
    r = potrf_resid(host2d(dA, n, n, n), A)
    assert r <= max(8 * U[prec], 4 * n * 2.0 ** -23), (prec, r)


@pytest.mark.parametrize("prec", ["bf16", "fp16", "bf16x3", "fp16x3"])
def test_sgetrf_mixed(hd, handle, torch_cuda, prec):
    n, nb = 1200, 256
    G = oracle.general_uniform(n, 1)
    dA = dev(torch_cuda, G)
    ipiv = torch_cuda.zeros(n, dtype=torch_cuda.int32, device="cuda")
    info = info_tensor(torch_cuda)
    st = hd.call("hdbf_sgetrf_mixed", handle.ptr, hd_mod.PREC[prec], ptr(dA), n, n, nb, ptr(ipiv),
                 ptr(info))
    torch_cuda.cuda.synchronize()
    assert st == 0 and int(info.item()) == 0
    piv = ipiv.cpu().numpy()
    assert np.all(piv >= np.arange(1, n + 1)) and np.all(piv <= n)
    r = oracle.getrf_residual_blas(host2d(dA, n, n, n), G, piv)
    growth_tol = 64 * U[prec]  # pivot growth on random matrices stays modest
    assert r <= max(growth_tol, 16 * n * 2.0 ** -23), (prec, r)


# nrhs <= 64 takes the wavefront solve (one launch per triangle and 32
# columns), wider right-hand sides the recursive GEMM solve; odd leading
# dimensions take the 4-byte tile copies, partial last blocks the zero fill.
@pytest.mark.parametrize("n,nrhs,pad", [(700, 16, 0), (64, 1, 0), (65, 3, 1), (1000, 33, 3),
                                        (2049, 64, 0), (513, 80, 1), (4096, 8, 0)])
def test_spotrs_sgetrs(hd, handle, torch_cuda, n, nrhs, pad):
    ld = n + pad
    A = oracle.spd_gram(n, 2)
    L = np.linalg.cholesky(A.astype(np.float64)).astype(np.float32)
    B = np.random.default_rng(3).standard_normal((n, nrhs)).astype(np.float32)
    dL, _ = padded(torch_cuda, L, ld)
    dB, _ = padded(torch_cuda, B, ld)
    st = hd.call("hdbf_spotrs", handle.ptr, ptr(dL), ld, n, nrhs, ptr(dB), ld)
    torch_cuda.cuda.synchronize()
    assert st == 0 and handle.device_errors() == 0
    X = host2d(dB, ld, ld, nrhs)
    want = np.linalg.solve(L.astype(np.float64) @ L.astype(np.float64).T, B.astype(np.float64))
    assert np.abs(X[:n] - want).max() <= 1e-4 * np.abs(want).max()
    if pad:
        assert np.all(np.isnan(X[n:]))
    G = oracle.general_uniform(n, 4) + np.float32(2.0) * np.eye(n, dtype=np.float32)
    lu, piv, info = oracle.lapack_sgetrf(G)
    dLU, _ = padded(torch_cuda, lu, ld)
    dP = dev(torch_cuda, piv)
    dB, _ = padded(torch_cuda, B, ld)
    st = hd.call("hdbf_sgetrs", handle.ptr, ptr(dLU), ld, n, ptr(dP), nrhs, ptr(dB), ld)
    torch_cuda.cuda.synchronize()
    assert st == 0 and handle.device_errors() == 0
    X = host2d(dB, ld, ld, nrhs)
    want = np.linalg.solve(G.astype(np.float64), B.astype(np.float64))
    assert np.abs(X[:n] - want).max() <= 1e-3 * np.abs(want).max()
    if pad:
        assert np.all(np.isnan(X[n:]))


def run_ir(hd, handle, torch, fn, A, B, prec, escalate=1, tol=1e-13, max_iter=30):
    n, nrhs = B.shape
    dA, dB = dev(torch, A), dev(torch, B)
    dX = torch.zeros(n * nrhs, dtype=torch.float64, device="cuda")
    info = hd_mod.IrInfo()
    st = hd.call(fn, handle.ptr, hd_mod.PREC[prec], escalate, ptr(dA), n, n, nrhs, ptr(dB), n,
                 ptr(dX), n, tol, max_iter, ctypes.byref(info))
    torch.cuda.synchronize()
    return st, host2d(dX, n, n, nrhs), info


@pytest.mark.parametrize("kappa,prec", [(1e2, "bf16"), (1e2, "fp16"), (1e4, "bf16"),
                                        (1e4, "fp16"), (1e6, "fp16x3"), (1e6, "bf16")])
def test_dposv_mixed_ir(hd, handle, torch_cuda, kappa, prec):
    n, nrhs = 1024, 16
    A = oracle.spd_kappa(n, kappa, 11)
    B = np.random.default_rng(12).standard_normal((n, nrhs))
    st, X, info = run_ir(hd, handle, torch_cuda, "hdbf_dposv_mixed", A, B, prec)
    assert st == 0, hd_mod.status_string(st)
    assert info.converged == 1, (info.backward_error, list(info.history[:info.iterations + 1]))
    assert oracle.backward_error(A, X, B) <= 1e-13
    assert info.backward_error <= 1e-13


@pytest.mark.parametrize("kappa,prec", [(1e2, "bf16"), (1e2, "fp16"), (1e4, "fp16"),
                                        (1e6, "fp16x3"), (1e6, "bf16")])
def test_dgesv_mixed_ir(hd, handle, torch_cuda, kappa, prec):
    n, nrhs = 1024, 16
    A = oracle.general_kappa(n, kappa, 21)
    B = np.random.default_rng(22).standard_normal((n, nrhs))
    st, X, info = run_ir(hd, handle, torch_cuda, "hdbf_dgesv_mixed", A, B, prec)
    assert st == 0, hd_mod.status_string(st)
    assert info.converged == 1, (info.backward_error, list(info.history[:info.iterations + 1]))
    assert oracle.backward_error(A, X, B) <= 1e-13


def run_gmres(hd, handle, torch, fn, A, B, prec, tol=1e-13, max_iter=10, max_inner=30,
              inner_tol=1e-4):
    n, nrhs = B.shape
    dA, dB = dev(torch, A), dev(torch, B)
    dX = torch.zeros(n * nrhs, dtype=torch.float64, device="cuda")
    info = hd_mod.IrInfo()
    st = hd.call(fn, handle.ptr, hd_mod.PREC[prec], ptr(dA), n, n, nrhs, ptr(dB), n, ptr(dX), n,
                 tol, max_iter, max_inner, inner_tol, ctypes.byref(info))
    torch.cuda.synchronize()
    return st, host2d(dX, n, n, nrhs), info


# GMRES-IR: FP64 GMRES preconditioned by the low-precision factors converges
# to the FP64 backward-error target where classical refinement needs
# escalation (BF16 LU) or stalls (kappa = 1e6 with FP32 factors), within the
# method's range kappa * u_factor <~ 1 (FP16 reaches kappa ~ 1e4, the split
# modes and FP32 kappa ~ 1e6).
@pytest.mark.parametrize("kappa,prec", [(1e2, "bf16"), (1e2, "fp16"), (1e4, "fp16"),
                                        (1e6, "fp16x3"), (1e6, "fp32")])
def test_dgesv_mixed_gmres(hd, handle, torch_cuda, kappa, prec):
    n, nrhs = 1024, 16
    A = oracle.general_kappa(n, kappa, 21)
    B = np.random.default_rng(22).standard_normal((n, nrhs))
    st, X, info = run_gmres(hd, handle, torch_cuda, "hdbf_dgesv_mixed_gmres", A, B, prec)
    assert st == 0, hd_mod.status_string(st)
    assert info.converged == 1, (info.backward_error, list(info.history[:info.iterations + 1]))
    assert oracle.backward_error(A, X, B) <= 1e-13
    assert info.inner_iterations >= 1 and info.factorizations == 1


@pytest.mark.parametrize("kappa,prec", [(1e2, "bf16"), (1e4, "fp16"), (1e6, "fp16x3")])
def test_dposv_mixed_gmres(hd, handle, torch_cuda, kappa, prec):
    n, nrhs = 1024, 5
    A = oracle.spd_kappa(n, kappa, 11)
    B = np.random.default_rng(12).standard_normal((n, nrhs))
    st, X, info = run_gmres(hd, handle, torch_cuda, "hdbf_dposv_mixed_gmres", A, B, prec)
    assert st == 0, hd_mod.status_string(st)
    assert info.converged == 1, (info.backward_error, list(info.history[:info.iterations + 1]))
    assert oracle.backward_error(A, X, B) <= 1e-13


def test_recursive_potrf_mixed_driver(hd, handle, torch_cuda):
    n = 1024
    A = oracle.spd_gram(n, 5)
    dA = dev(torch_cuda, A)
    info = info_tensor(torch_cuda)
    hd.call("recursive_potrf_mixed_driver", handle.ptr, None, ptr(dA), n, n, 256, ptr(info))
    torch_cuda.cuda.synchronize()
    handle.check()
    assert int(info.item()) == 0
    assert potrf_resid(host2d(dA, n, n, n), A) <= 8 * U["fp16"]


def test_batched_syrk_and_trsm_mixed(hd, handle, torch_cuda):
    n, k = 600, 200
    rng = np.random.default_rng(9)
    A = rng.uniform(-1, 1, (n, k)).astype(np.float32)
    C = rng.uniform(-1, 1, (n, n)).astype(np.float32)
    dA, dC = dev(torch_cuda, A), dev(torch_cuda, C)
    hd.call("batched_syrk_bottom_up_mixed", handle.ptr, None, ptr(dA), n, ptr(dC), n, n, k, 128)
    torch_cuda.cuda.synchronize()
    handle.check()
    a16 = A.astype(np.float16).astype(np.float64)
    want = C.astype(np.float64) - a16 @ a16.T
    got = host2d(dC, n, n, n)
    lo = np.tril_indices(n)
    assert np.abs(got[lo] - want[lo]).max() <= 1e-4 * np.abs(want).max()
    m = 300
    L = np.tril(rng.uniform(-1, 1, (m, m))) * 0.05
    L[np.diag_indices(m)] = 1.0 + rng.uniform(0, 1, m)
    L = L.astype(np.float32)
    Bm = rng.uniform(-1, 1, (n, m)).astype(np.float32)
    dL, dB = dev(torch_cuda, L), dev(torch_cuda, Bm)
    hd.call("recursive_trsm_mixed", handle.ptr, ptr(dL), m, ptr(dB), n, n, m, 64)
    torch_cuda.cuda.synchronize()
    handle.check()
    want = np.linalg.solve(L.astype(np.float64), Bm.astype(np.float64).T).T
    got = host2d(dB, n, n, m)
    assert np.abs(got - want).max() <= 2e-2 * np.abs(want).max()


def test_wave_solve_repeated_launches(hd, handle, torch_cuda):
    """Wavefront solves of different orders back to back: the ready flags and
    solution copies an earlier (larger) launch left behind are never taken
    for the current ones; the repeated results are bit-identical and match
    the FP64 solution."""
    out = {}
    for rep in range(2):
        for n, nrhs in ((4096, 16), (700, 5), (4096, 16), (1500, 32)):
            A = oracle.spd_gram(n, 9)
            L = np.linalg.cholesky(A.astype(np.float64)).astype(np.float32)
            B = np.random.default_rng(n + nrhs).standard_normal((n, nrhs)).astype(np.float32)
            dL = dev(torch_cuda, L)
            dB = dev(torch_cuda, B)
            st = hd.call("hdbf_spotrs", handle.ptr, ptr(dL), n, n, nrhs, ptr(dB), n)
            torch_cuda.cuda.synchronize()
            assert st == 0 and handle.device_errors() == 0
            X = host2d(dB, n, n, nrhs)
            if (n, nrhs) in out:
                np.testing.assert_array_equal(X, out[(n, nrhs)])
            else:
                want = np.linalg.solve(L.astype(np.float64) @ L.astype(np.float64).T,
                                       B.astype(np.float64))
                assert np.abs(X - want).max() <= 1e-4 * np.abs(want).max()
                out[(n, nrhs)] = X


def run_auto(hd, handle, torch, fn, A, B, prec, tol=1e-13, max_iter=30):
    n, nrhs = B.shape
    dA, dB = dev(torch, A), dev(torch, B)
    dX = torch.zeros(n * nrhs, dtype=torch.float64, device="cuda")
    info = hd_mod.IrInfo()
    st = hd.call(fn, handle.ptr, hd_mod.PREC[prec], ptr(dA), n, n, nrhs, ptr(dB), n, ptr(dX), n,
                 tol, max_iter, ctypes.byref(info))
    torch.cuda.synchronize()
    return st, host2d(dX, n, n, nrhs), info


# Adaptive refinement: classical corrections while they halve the backward
# error, then GMRES-IR, then a higher factorization precision.  A
# well-conditioned SPD system finishes on classical steps alone; an
# ill-conditioned general one (kappa = 1e6 is beyond BF16 factors, kappa *
# u_bf16 ~ 4e3) needs GMRES and at least one refactorization, and still
# reaches the FP64 target.
def test_dposv_mixed_auto_classical_only(hd, handle, torch_cuda):
    n, nrhs = 1024, 8
    A = oracle.spd_kappa(n, 1e2, 11)
    B = np.random.default_rng(12).standard_normal((n, nrhs))
    st, X, info = run_auto(hd, handle, torch_cuda, "hdbf_dposv_mixed_auto", A, B, "fp16")
    assert st == 0, hd_mod.status_string(st)
    assert info.converged == 1 and info.inner_iterations == 0 and info.factorizations == 1
    assert info.final_precision == hd_mod.PREC["fp16"]
    assert oracle.backward_error(A, X, B) <= 1e-13


@pytest.mark.parametrize("prec", ["bf16", "fp16"])
def test_dgesv_mixed_auto_escalates(hd, handle, torch_cuda, prec):
    n, nrhs = 1024, 8
    A = oracle.general_kappa(n, 1e6, 21)
    B = np.random.default_rng(22).standard_normal((n, nrhs))
    st, X, info = run_auto(hd, handle, torch_cuda, "hdbf_dgesv_mixed_auto", A, B, prec)
    assert st == 0, hd_mod.status_string(st)
    assert info.converged == 1, (info.backward_error, list(info.history[:info.iterations + 1]),
                                 info.final_precision, info.factorizations)
    assert oracle.backward_error(A, X, B) <= 1e-13
    # the LU escalation order: BF16 goes to the FP16 split (more significant bits)
    chain = [prec, "fp16x3", "fp32"]
    assert info.final_precision == hd_mod.PREC[chain[info.factorizations - 1]], \
        (info.final_precision, info.factorizations)
