"""Host-side helpers for the batched factor-and-solve entry point
(hdbf_batched_factor_solve): packs many small systems into one device
allocation, builds the device pointer / size / order arrays, and generates the
seeded batch workloads (SPD G G^T/n + I with G from the counter-based U[-1,1)
generator, general U[-1,1) matrices, N(0,1) right-hand sides)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import lib


class DeviceBatch:
    """Packed batch on the GPU.  ops[i] = 0 (Cholesky) or 1 (LU)."""

    def __init__(self, torch, ops, ns):
        self.torch = torch
        self.ops = np.asarray(ops, dtype=np.int32)
        self.ns = np.asarray(ns, dtype=np.int32)
        self.count = len(self.ns)
        sizes = self.ns.astype(np.int64) ** 2
        self.offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        self.roffsets = np.concatenate([[0], np.cumsum(self.ns)[:-1]]).astype(np.int64)
        dev = "cuda"
        self.A = torch.zeros(int(sizes.sum()), dtype=torch.float32, device=dev)
        self.b = torch.zeros(int(self.ns.sum()), dtype=torch.float32, device=dev)
        self.ipiv_buf = torch.zeros(int(self.ns.sum()), dtype=torch.int32, device=dev)
        self.info = torch.zeros(self.count, dtype=torch.int32, device=dev)
        self.queue = torch.zeros(1, dtype=torch.int32, device=dev)
        a0, b0, p0 = self.A.data_ptr(), self.b.data_ptr(), self.ipiv_buf.data_ptr()
        self.d_A = torch.tensor(a0 + 4 * self.offsets, dtype=torch.int64, device=dev)
        self.d_b = torch.tensor(b0 + 4 * self.roffsets, dtype=torch.int64, device=dev)
        self.d_ipiv = torch.tensor(p0 + 4 * self.roffsets, dtype=torch.int64, device=dev)
        self.d_n = torch.tensor(self.ns, dtype=torch.int32, device=dev)
        self.d_lda = torch.tensor(self.ns, dtype=torch.int32, device=dev)
        self.d_op = torch.tensor(self.ops, dtype=torch.int32, device=dev)
        work = np.where(self.ops == 0, self.ns.astype(np.float64) ** 3 / 3.0,
                        2.0 * self.ns.astype(np.float64) ** 3 / 3.0)
        self.d_order = torch.tensor(np.argsort(-work, kind="stable").astype(np.int32), device=dev)

    def flops(self) -> float:
        n = self.ns.astype(np.float64)
        fac = np.where(self.ops == 0, n ** 3 / 3.0, 2.0 * n ** 3 / 3.0)
        return float((fac + 2.0 * n ** 2).sum())

    def matrix(self, i):
        n = int(self.ns[i])
        o = int(self.offsets[i])
        return self.A[o:o + n * n].view(n, n).t()  # column-major view

    def rhs(self, i):
        o, n = int(self.roffsets[i]), int(self.ns[i])
        return self.b[o:o + n]

    def pivots(self, i):
        o, n = int(self.roffsets[i]), int(self.ns[i])
        return self.ipiv_buf[o:o + n]

    def run(self, handle, variant):
        P = ctypes.c_void_p
        return lib().hdbf_batched_factor_solve(
            handle.ptr, int(variant), self.count, P(self.d_order.data_ptr()),
            P(self.d_op.data_ptr()), P(self.d_n.data_ptr()), P(self.d_lda.data_ptr()),
            P(self.d_A.data_ptr()), P(self.d_b.data_ptr()), P(self.d_ipiv.data_ptr()),
            P(self.info.data_ptr()), P(self.queue.data_ptr()))


def config3_sizes(n_spd=4096, n_gen=2048, seed=3):
    """Sizes of the batched workload: SPD n ~ U[16, 512], general n ~ U[32, 768]."""
    rng = np.random.default_rng(seed)
    ns_spd = rng.integers(16, 513, size=n_spd)
    ns_gen = rng.integers(32, 769, size=n_gen)
    ops = np.concatenate([np.zeros(n_spd, np.int32), np.ones(n_gen, np.int32)])
    return ops, np.concatenate([ns_spd, ns_gen]).astype(np.int32)


def fill_batch(torch, handle, batch: DeviceBatch, seed=3):
    """Seeded inputs on the device: SPD A = G G^T / n + I (FP64, rounded to
    FP32; G from the counter-based generator at offset = packed position),
    general A iid U[-1,1), right-hand sides N(0,1).  Keeps pristine copies."""
    L = lib()
    st = L.hdbf_fill_uniform(handle.ptr, ctypes.c_void_p(batch.A.data_ptr()), batch.A.numel(),
                             seed, 0)
    assert st == 0
    for i in range(batch.count):
        if batch.ops[i] == 0:
            n = int(batch.ns[i])
            G = batch.matrix(i).double()
            A = G @ G.t() / n
            A.diagonal().add_(1.0)
            batch.matrix(i).copy_((0.5 * (A + A.t())).float())
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    batch.b.copy_(torch.randn(batch.b.numel(), generator=g, device="cuda"))
    batch.A0 = batch.A.clone()
    batch.b0 = batch.b.clone()


def restore(batch: DeviceBatch):
    batch.A.copy_(batch.A0)
    batch.b.copy_(batch.b0)
