"""GPU tests of the tensor-core (tcgen05) mixed-precision GEMM through the
reference's launch_mixed_gemm entry point: FP16-rounded operands, FP32
accumulation, FP32 C.  Reference: the same FP16-rounded operands multiplied
in FP64 on the host."""
import numpy as np
import pytest

from tests.common import dev, host2d, ptr

pytestmark = pytest.mark.gpu

NONE, TRANS = 111, 112


def rnd(shape, seed):
    return np.random.default_rng(seed).uniform(-1, 1, size=shape).astype(np.float32)


@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (1, 1, 1), (300, 200, 77), (1000, 513, 1000),
                                   (4096, 4096, 1024), (257, 129, 4100)])
@pytest.mark.parametrize("ta,tb", [(NONE, TRANS), (NONE, NONE), (TRANS, NONE), (TRANS, TRANS)])
def test_mixed_gemm_matches_fp64_of_rounded_inputs(hd, handle, torch_cuda, m, n, k, ta, tb):
    A = rnd((m, k) if ta == NONE else (k, m), 1)
    B = rnd((k, n) if tb == NONE else (n, k), 2)
    C = rnd((m, n), 3)
    alpha, beta = np.float32(-1.0), np.float32(1.0)
    dA, dB, dC = dev(torch_cuda, A), dev(torch_cuda, B), dev(torch_cuda, C)
    stream = torch_cuda.cuda.current_stream().cuda_stream
    hd.call("launch_mixed_gemm", handle.ptr, stream, ta, tb, m, n, k, alpha, ptr(dA), A.shape[0],
            ptr(dB), B.shape[0], beta, ptr(dC), m)
    torch_cuda.cuda.synchronize()
    handle.check("launch_mixed_gemm")
    assert handle.device_errors() == 0
    a16 = A.astype(np.float16).astype(np.float64)
    b16 = B.astype(np.float16).astype(np.float64)
    opA = a16 if ta == NONE else a16.T
    opB = b16 if tb == NONE else b16.T
    want = beta * C.astype(np.float64) + alpha * (opA @ opB)
    got = host2d(dC, m, m, n)
    # exact FP16 products, FP32 accumulation over k terms of magnitude <= 1
    tol = 4 * max(k, 16) * 2.0 ** -23 * max(1.0, np.abs(want).max())
    assert np.abs(got - want).max() <= tol


def test_mixed_gemm_alpha_beta(hd, handle, torch_cuda):
    m, n, k = 200, 150, 96
    A, B, C = rnd((m, k), 4), rnd((k, n), 5), rnd((m, n), 6)
    dA, dB, dC = dev(torch_cuda, A), dev(torch_cuda, B), dev(torch_cuda, C)
    stream = torch_cuda.cuda.current_stream().cuda_stream
    hd.call("launch_mixed_gemm", handle.ptr, stream, NONE, NONE, m, n, k, np.float32(0.5),
            ptr(dA), m, ptr(dB), k, np.float32(-2.0), ptr(dC), m)
    torch_cuda.cuda.synchronize()
    want = -2.0 * C.astype(np.float64) + 0.5 * (A.astype(np.float16).astype(np.float64)
                                                @ B.astype(np.float16).astype(np.float64))
    assert np.abs(host2d(dC, m, m, n) - want).max() <= 1e-4 * np.abs(want).max()
