"""Shared helpers for the GPU parity tests (device buffers via torch)."""
from __future__ import annotations

import ctypes

import numpy as np

import oracle

P = ctypes.c_void_p


def dev(torch, arr, dtype=None):
    """Host numpy (2-D column-major view or 1-D) -> flat device tensor."""
    a = np.asarray(arr)
    if a.ndim == 2:
        a = a.ravel(order="F")
    t = torch.from_numpy(np.ascontiguousarray(a if dtype is None else a.astype(dtype)))
    return t.cuda()


def padded(torch, A2d, lda, fill=np.nan, dtype=np.float32):
    """Column-major n x n matrix stored with leading dimension lda (padding = fill)."""
    n = A2d.shape[0]
    buf = np.full((lda, A2d.shape[1]), fill, dtype=dtype)
    buf[:n, :] = A2d
    return dev(torch, buf), buf


def host2d(t, lda, rows, cols):
    """Flat device tensor with leading dimension lda -> rows x cols numpy."""
    flat = t.detach().cpu().numpy()
    return flat.reshape(cols, lda).T[:rows, :cols].copy()


def ptr(t):
    return P(t.data_ptr())


def info_tensor(torch):
    return torch.full((1,), 12345, dtype=torch.int32, device="cuda")


def potrf_check(L2d, A2d):
    """Scaled CPU FP64 residual (C oracle) of a Cholesky factor."""
    n = A2d.shape[0]
    r = oracle.potrf_residual(np.asfortranarray(L2d, dtype=np.float32).ravel(order="F"),
                              np.asfortranarray(A2d, dtype=np.float32).ravel(order="F"), n, n)
    return oracle.scaled(r, n)


def getrf_check(LU2d, A2d, ipiv, pivoting=True):
    n = A2d.shape[0]
    r = oracle.getrf_residual(np.asfortranarray(LU2d, dtype=np.float32).ravel(order="F"),
                              np.asfortranarray(A2d, dtype=np.float32).ravel(order="F"),
                              None if ipiv is None else np.asarray(ipiv, dtype=np.int32), n, n,
                              pivoting=pivoting)
    return oracle.scaled(r, n)
