"""Cholesky panel fallback of the mixed-precision factorization: a panel whose
diagonal block meets a non-positive pivot after the low-precision trailing
updates is rebuilt in FP32 from the original matrix and factored again
(hdbf_spotrf_mixed, hdbf_mixed_fallback_panels, hdbf_ir_info.fallback_panels).

* A matrix that is not positive definite keeps LAPACK spotrf's info (the
  FP32 panel fails too).
* SPD matrices whose FP16 trailing updates break the factorization: the
  fallback rebuilds the failing panels, the factorization completes
  (info 0) with a residual at the level of the 16-bit updates, and FP64
  refinement (GMRES-IR) still reaches a backward error <= 1e-13 -- with no
  refactorization at a higher precision (factorizations == 1)."""
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


def test_fp16_fallback_rebuilds_failing_panels(hd, handle, torch_cuda):
    torch = torch_cuda
    n, nb = 2048, 256
    seen = []
    for kappa in (1e3, 1e4, 1e5):
        A64 = spd(torch, n, kappa, seed=int(kappa))
        st, dA, info, cnt = mixed_potrf(hd, handle, torch, A64.float(), "fp16", nb)
        assert st == 0 and handle.device_errors() == 0
        seen.append((kappa, info, cnt))
        if cnt > 0 and info == 0:
            L = torch.tril(dA.view(n, n).t().double())
            r = float(torch.linalg.matrix_norm(A64 - L @ L.t()) / torch.linalg.matrix_norm(A64))
            assert r <= 5e-3, (kappa, r)  # FP16-update level, not garbage
    assert any(c > 0 and i == 0 for _, i, c in seen), seen
    # refinement on the same family: the fallback keeps the first factorization usable
    kappa = max(k for k, i, c in seen if c > 0 and i == 0)
    A64 = spd(torch, n, kappa, seed=int(kappa))
    B = torch.randn(n, 4, dtype=torch.float64, device="cuda")
    dA = A64.t().contiguous().reshape(-1)
    dB = B.t().contiguous().reshape(-1)
    dX = torch.zeros_like(dB)
    info = hd_mod.IrInfo()
    st = hd.call("hdbf_dposv_mixed_gmres", handle.ptr, hd_mod.PREC["fp16"], ptr(dA), n, n, 4,
                 ptr(dB), n, ptr(dX), n, ctypes.c_double(1e-13), 10, 40, ctypes.c_double(1e-4),
                 ctypes.byref(info))
    assert st == 0
    assert info.fallback_panels > 0 and info.factorizations == 1 and info.info == 0
    assert info.converged == 1 and info.backward_error <= 1e-13, info.backward_error
