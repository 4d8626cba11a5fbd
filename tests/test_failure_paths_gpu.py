"""Failure paths on the GPU, in forms that fault or hang nothing.

* Bounded waits: the handle's wait limit is set to a single poll, so the
  grid-wide exchanges of the GETRF panel kernel and the grid barriers of the
  diagonal-block Cholesky kernel give up at once; the call must come back with
  HDBF_STATUS_TIMEOUT from hdbf_check_device_errors, and the next call on the
  same handle (default limit restored) must factor correctly.
* Corrupt pivots handed to launch_apply_getrf_panel_pivots (a pivot row above
  its own row): the composition rejects them and moves no row.
* NaN inputs: POTRF reports the first NaN / non-positive pivot as the
  reference LAPACK xPOTRF does; GETRF completes with no device error and the NaN reaches the
  factors (non-finite oracle residual)."""
import ctypes

import numpy as np
import pytest

import oracle
from tests.common import dev, host2d, info_tensor, padded, ptr
from tests.test_getrf_gpu import run_getrf

pytestmark = pytest.mark.gpu

HDBF_STATUS_TIMEOUT = 6


def test_wait_limit_timeout_in_getrf_panel(hd, handle, torch_cuda):
    n = 2048
    G = oracle.general_uniform(n, 1)
    handle.set_panel_kernel(1)  # grid-wide publish-and-poll panel kernel
    try:
        handle.set_wait_limit(1)
        run_getrf(hd, handle, torch_cuda, G, "double_blocked_getrf", outer=1024, inner=256)
        assert handle.device_errors() == HDBF_STATUS_TIMEOUT
        assert handle.device_errors() == 0  # read once, then cleared
        handle.set_wait_limit(0)
        _, LU, ipiv, info = run_getrf(hd, handle, torch_cuda, G, "double_blocked_getrf",
                                      outer=1024, inner=256)
        handle.check()
        assert handle.device_errors() == 0 and info == 0
        assert oracle.pivot_agreement(G, oracle.lapack_sgetrf(G)[1], ipiv)["near_tie"]
        assert oracle.scaled(oracle.getrf_residual_tiled(LU[:n], G, ipiv), n) <= 10.0
    finally:
        handle.set_wait_limit(0)
        handle.set_panel_kernel(0)


def test_wait_limit_timeout_in_diagonal_block(hd, handle, torch_cuda):
    n = 1024
    A = oracle.spd_gram(n, 0)
    dA0 = dev(torch_cuda, A)
    info = info_tensor(torch_cuda)
    try:
        handle.set_wait_limit(1)
        dA = dA0.clone()
        # inner block 512: one cooperative diagonal-block launch per block
        hd.call("double_blocked_potrf", handle.ptr, ptr(dA), n, n, 1024, 512, ptr(info))
        torch_cuda.cuda.synchronize()
        assert handle.device_errors() == HDBF_STATUS_TIMEOUT
        handle.set_wait_limit(0)
        dA = dA0.clone()
        hd.call("double_blocked_potrf", handle.ptr, ptr(dA), n, n, 1024, 512, ptr(info))
        torch_cuda.cuda.synchronize()
        handle.check()
        assert handle.device_errors() == 0 and int(info.item()) == 0
        L = host2d(dA, n, n, n)
        assert oracle.scaled(oracle.potrf_residual_tiled(L, A), n) <= 10.0
    finally:
        handle.set_wait_limit(0)


def test_corrupt_panel_pivots_move_nothing(hd, handle, torch_cuda):
    n, panel, size = 300, 40, 50
    rng = np.random.default_rng(0)
    A = rng.standard_normal((n, n)).astype(np.float32)
    piv = np.array([rng.integers(o + 1, n - panel + 1) for o in range(size)], dtype=np.int32)
    piv[7] = 3  # row 7 of the panel may not swap with panel row 2
    dA = dev(torch_cuda, A)
    dp = dev(torch_cuda, piv)
    stream = torch_cuda.cuda.current_stream().cuda_stream
    hd.call("launch_apply_getrf_panel_pivots", ptr(dA), n, n, panel, size, ptr(dp), stream)
    torch_cuda.cuda.synchronize()
    np.testing.assert_array_equal(host2d(dA, n, n, n), A)


def test_nan_diagonal_potrf_info(hd, handle, torch_cuda):
    """A NaN diagonal stops the factorization with info = its column, as the
    reference LAPACK xPOTRF does (`ajj <= 0 or isnan(ajj)`); host OpenBLAS
    spotrf does not test for NaN and returns 0, so the expected value is the
    reference LAPACK rule, checked on the same matrix with the NaN replaced by
    a negative value (which both treat alike)."""
    n = 1024
    A = oracle.spd_gram(n, 0)
    A[300, 300] = np.nan
    dA, _ = padded(torch_cuda, A, n)
    info = info_tensor(torch_cuda)
    hd.call("double_blocked_potrf_kblocked_syrk", handle.ptr, ptr(dA), n, n, 512, 128, 0,
            ptr(info))
    torch_cuda.cuda.synchronize()
    assert handle.device_errors() == 0
    A2 = A.copy()
    A2[300, 300] = -1.0
    _, info_l = oracle.lapack_spotrf(A2)
    assert int(info.item()) == info_l == 301


def test_nan_entry_getrf_completes(hd, handle, torch_cuda):
    n = 1024
    G = oracle.general_uniform(n, 2)
    G[500, 100] = np.nan
    _, LU, ipiv, info = run_getrf(hd, handle, torch_cuda, G, "double_blocked_getrf", outer=512,
                                  inner=128)
    assert handle.device_errors() == 0
    assert info >= 0
    assert np.all((ipiv >= np.arange(1, n + 1)) & (ipiv <= n))  # valid LAPACK pivots
    assert np.isnan(LU).any()
    assert np.isinf(oracle.getrf_residual_tiled(LU[:n], G, ipiv))
