"""Cholesky panel fallback of the mixed-precision factorization: a panel whose
diagonal block meets a non-positive pivot after the low-precision trailing
updates is rebuilt in FP32 from the original matrix and factored again
(hdbf_spotrf_mixed, hdbf_mixed_fallback_panels, hdbf_ir_info.fallback_panels).

* A matrix that is not positive definite keeps LAPACK spotrf's info (the
  FP32 panel fails too).
* An SPD matrix whose FP16 trailing update breaks one panel: the fallback
  rebuilds that panel, the factorization completes (info 0) with an FP32-level
  residual, and FP64 refinement (GMRES-IR) reaches a backward error <= 1e-13
  with that one factorization (no refactorization at a higher precision)."""
import ctypes

import numpy as np
import pytest

import hygondoubleblockedfactorizations_b200 as hd_mod
import oracle
from tests.common import info_tensor, ptr

pytestmark = pytest.mark.gpu


def spd(torch, n, kappa, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    Q, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    lam = torch.logspace(0.0, float(np.log10(kappa)), n, dtype=torch.float64, device="cuda")
    A = (Q * lam) @ Q.t()
    return 0.5 * (A + A.t())


def mixed_potrf(hd, handle, torch, A32, prec, nb):
    n = A32.shape[0]
    dA = A32.t().contiguous().reshape(-1).clone()  # column-major storage
    info = info_tensor(torch)
    st = hd.call("hdbf_spotrf_mixed", handle.ptr, hd_mod.PREC[prec], ptr(dA), n, n, nb, ptr(info))
    torch.cuda.synchronize()
    cnt = ctypes.c_int(-1)
    assert hd.lib().hdbf_mixed_fallback_panels(handle.ptr, ctypes.byref(cnt)) == 0
    return st, dA, int(info.item()), cnt.value


@pytest.mark.parametrize("prec", ["bf16", "fp16"])
def test_indefinite_keeps_lapack_info(hd, handle, torch_cuda, prec):
    n = 1024
    A = oracle.spd_gram(n, 0)
    A[700, 700] = -5.0
    _, info_l = oracle.lapack_spotrf(A)
    st, _, info, cnt = mixed_potrf(hd, handle, torch_cuda,
                                   torch_cuda.from_numpy(np.ascontiguousarray(A)).cuda(), prec, 256)
    assert st == 0 and handle.device_errors() == 0
    assert info == info_l == 701
    assert cnt >= 1  # the panel holding column 701 took the fallback, which failed too


def fallback_matrix(b, delta, seed):
    """A = [[I, C, 0], [C^T, C^T C + delta I, 0], [0, 0, I]] (blocks b x b, C iid
    U[-1,1)), formed in FP64 and rounded to FP32.  Its second diagonal block's
    Schur complement is delta I.  The FP16 rounding of the panel C^T in the
    trailing update moves its smallest eigenvalue to about -0.04 (first
    attempt fails); recomputed in FP32 from the original with the panel's
    accurate (BF16x3 TRSM) factor it stays near +0.009 (checked on the CPU
    with the same roundings)."""
    rng = np.random.default_rng(seed)
    C = rng.uniform(-1, 1, size=(b, b))
    n = 3 * b
    A = np.eye(n)
    A[:b, b:2 * b] = C
    A[b:2 * b, :b] = C.T
    A[b:2 * b, b:2 * b] = C.T @ C + delta * np.eye(b)
    return A.astype(np.float32), A


def test_fp16_fallback_rebuilds_failing_panel(hd, handle, torch_cuda):
    torch = torch_cuda
    b, delta = 256, 1e-2
    A32, A64 = fallback_matrix(b, delta, 5)
    n = A32.shape[0]
    _, info_l = oracle.lapack_spotrf(A32)
    assert info_l == 0  # positive definite in FP32
    At = torch.from_numpy(np.ascontiguousarray(A32)).cuda()
    st, dA, info, cnt = mixed_potrf(hd, handle, torch, At, "fp16", b)
    assert st == 0 and handle.device_errors() == 0
    assert cnt == 1 and info == 0, (cnt, info)  # the second panel was rebuilt in FP32
    L = torch.tril(dA.view(n, n).t().double())
    Ad = torch.from_numpy(A64).cuda()
    r = float(torch.linalg.matrix_norm(Ad - L @ L.t()) / torch.linalg.matrix_norm(Ad))
    assert r <= 5e-5, r
    # FP64 refinement (GMRES-IR: A is ill-conditioned, kappa ~ 1e7) with the
    # same factorization: no refactorization at a higher precision
    B = torch.randn(n, 4, dtype=torch.float64, device="cuda")
    dB = B.t().contiguous().reshape(-1)
    dX = torch.zeros_like(dB)
    ir = hd_mod.IrInfo()
    st = hd.call("hdbf_dposv_mixed_gmres", handle.ptr, hd_mod.PREC["fp16"],
                 ptr(Ad.t().contiguous().reshape(-1)), n, n, 4, ptr(dB), n, ptr(dX), n,
                 ctypes.c_double(1e-13), 10, 60, ctypes.c_double(1e-6), ctypes.byref(ir))
    assert st == 0
    assert ir.fallback_panels == 1 and ir.factorizations == 1 and ir.info == 0
    assert ir.converged == 1 and ir.backward_error <= 1e-13, ir.backward_error
