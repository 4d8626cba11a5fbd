"""Both tensor-core GEMM kernels behind the mixed-precision updates, through
the C ABI: the persistent kernel (128 x 256 tiles, two TMEM accumulators,
the default) and the one-tile-per-CTA kernel (128 x 128), chosen per handle
with HDBF_TC_KERNEL at handle creation.  Each must match the FP64 product of
the FP16-rounded operands for plain updates (launch_mixed_gemm) and for
lower-triangle updates (batched_syrk_bottom_up_mixed: only entries with
row >= col change), at shapes with ragged edges, several tiles per CTA,
more tiles than SMs, and a partial last band of 256 columns."""
import os

import numpy as np
import pytest

from tests.common import dev, host2d, ptr

pytestmark = pytest.mark.gpu

NONE, TRANS = 111, 112


def make_handle(hd, torch, kernel):
    old = os.environ.get("HDBF_TC_KERNEL")
    os.environ["HDBF_TC_KERNEL"] = str(kernel)
    try:
        return hd.Handle(torch.cuda.current_stream().cuda_stream)
    finally:
        if old is None:
            del os.environ["HDBF_TC_KERNEL"]
        else:
            os.environ["HDBF_TC_KERNEL"] = old


def rnd(shape, seed):
    return np.random.default_rng(seed).uniform(-1, 1, size=shape).astype(np.float32)


def r16(x):
    return x.astype(np.float16).astype(np.float64)


@pytest.mark.parametrize("kernel", [0, 1])
@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (300, 700, 77), (5000, 1000, 520),
                                   (2048, 8192, 256), (130, 260, 1030)])
def test_plain_update(hd, torch_cuda, kernel, m, n, k):
    h = make_handle(hd, torch_cuda, kernel)
    try:
        A, B, C = rnd((m, k), 1), rnd((n, k), 2), rnd((m, n), 3)
        dA, dB, dC = dev(torch_cuda, A), dev(torch_cuda, B), dev(torch_cuda, C)
        stream = torch_cuda.cuda.current_stream().cuda_stream
        hd.call("launch_mixed_gemm", h.ptr, stream, NONE, TRANS, m, n, k, np.float32(-1.0),
                ptr(dA), m, ptr(dB), n, np.float32(1.0), ptr(dC), m)
        torch_cuda.cuda.synchronize()
        h.check("launch_mixed_gemm")
        assert h.device_errors() == 0
        want = C.astype(np.float64) - r16(A) @ r16(B).T
        tol = 4 * max(k, 16) * 2.0 ** -23 * max(1.0, np.abs(want).max())
        assert np.abs(host2d(dC, m, m, n) - want).max() <= tol
    finally:
        torch_cuda.cuda.synchronize()
        h.close()


@pytest.mark.parametrize("kernel", [0, 1])
@pytest.mark.parametrize("n,k", [(256, 64), (1000, 300), (3000, 1024), (600, 40)])
def test_lower_update(hd, torch_cuda, kernel, n, k):
    h = make_handle(hd, torch_cuda, kernel)
    try:
        A, C = rnd((n, k), 4), rnd((n, n), 5)
        dA, dC = dev(torch_cuda, A), dev(torch_cuda, C)
        hd.call("batched_syrk_bottom_up_mixed", h.ptr, None, ptr(dA), n, ptr(dC), n, n, k, 128)
        torch_cuda.cuda.synchronize()
        h.check("batched_syrk_bottom_up_mixed")
        assert h.device_errors() == 0
        got = host2d(dC, n, n, n)
        want = C.astype(np.float64) - r16(A) @ r16(A).T
        low = np.tril(np.ones((n, n), dtype=bool))
        np.testing.assert_array_equal(got[~low], C[~low])  # strictly upper part untouched
        tol = 4 * max(k, 16) * 2.0 ** -23 * max(1.0, np.abs(want).max())
        assert np.abs(got[low] - want[low]).max() <= tol
    finally:
        torch_cuda.cuda.synchronize()
        h.close()
