"""GPU parity tests for the Cholesky path, called through the C ABI.

Oracle: the C restatement of the reference's CPU FP64 residual (scaled by
n * eps32, eps32 = 2**-23; bound 10) next to host LAPACK spotrf's residual on
the same input, plus element-wise agreement with LAPACK's factor."""
import numpy as np
import pytest

import oracle
from tests.common import P, dev, host2d, info_tensor, padded, potrf_check, ptr

pytestmark = pytest.mark.gpu

BOUND = 10.0  # scaled residual bound from the workload definition


def run_potrf(hd, handle, torch, A2d, fn, lda=None, **kw):
    n = A2d.shape[0]
    lda = lda or n
    dA, _ = padded(torch, A2d, lda)
    info = info_tensor(torch)
    h = handle.ptr
    nb, b = kw.get("nb", 0), kw.get("b", 0)
    if fn == "double_blocked_potrf":
        hd.call(fn, h, ptr(dA), lda, n, nb, b, ptr(info))
    elif fn == "double_blocked_potrf_dbtrsm":
        hd.call(fn, h, ptr(dA), lda, n, nb, b, ptr(info))
    elif fn in ("double_blocked_potrf_kblocked_syrk", "double_blocked_potrf_kblocked_syrk_adaptive_gemm"):
        hd.call(fn, h, ptr(dA), lda, n, nb, b, kw.get("tk", 0), ptr(info))
    elif fn == "double_blocked_potrf_kblocked_syrk_adaptive_gemm_configured":
        hd.call(fn, h, ptr(dA), lda, n, nb, b, kw.get("tk", 0), kw.get("mt", 256),
                kw.get("mthr", 0), kw.get("kthr", 0), ptr(info))
    elif fn == "blocked_right_looking_potrf":
        hd.call(fn, h, ptr(dA), lda, n, nb, ptr(info))
    elif fn in ("recursive_potrf", "recursive_potrf_tiled_trsm"):
        hd.call(fn, h, None, ptr(dA), lda, n, nb, ptr(info))
    else:
        raise ValueError(fn)
    torch.cuda.synchronize()
    handle.check(fn)
    assert handle.device_errors() == 0
    return host2d(dA, lda, lda, n), int(info.item())


VARIANTS = [
    ("double_blocked_potrf", {}),
    ("double_blocked_potrf_dbtrsm", {}),
    ("double_blocked_potrf_kblocked_syrk", {"tk": 384}),
    ("double_blocked_potrf_kblocked_syrk_adaptive_gemm", {"tk": 512}),
    ("double_blocked_potrf_kblocked_syrk_adaptive_gemm_configured", {"tk": 256, "mt": 300, "mthr": 100, "kthr": 64}),
    ("blocked_right_looking_potrf", {}),
    ("recursive_potrf", {}),
    ("recursive_potrf_tiled_trsm", {}),
]


@pytest.mark.parametrize("fn,kw", VARIANTS, ids=[v[0] for v in VARIANTS])
def test_config0_all_variants(hd, handle, torch_cuda, fn, kw):
    """n=2048, outer 512, inner 64 (recursive: leaf 256)."""
    n = 2048
    A = oracle.spd_gram(n, 0)
    nb = 256 if fn.startswith("recursive") else 512
    L, info = run_potrf(hd, handle, torch_cuda, A, fn, nb=nb, b=64, **kw)
    assert info == 0
    ours = potrf_check(np.tril(L[:n]), A)
    Lref, linfo = oracle.lapack_spotrf(A)
    ref = potrf_check(np.tril(Lref), A)
    assert linfo == 0
    assert ours <= BOUND, (ours, ref)
    # the factor itself agrees with LAPACK's to FP32 rounding (well-conditioned A)
    d = np.abs(np.tril(L[:n]).astype(np.float64) - np.tril(Lref).astype(np.float64)).max()
    assert d <= 1e-4 * np.abs(Lref).max()


@pytest.mark.parametrize("n,nb,b", [(1, 0, 0), (2, 1, 1), (3, 2, 1), (17, 8, 3), (63, 64, 64),
                                    (64, 32, 16), (65, 64, 64), (127, 50, 7), (130, 128, 64),
                                    (257, 100, 33), (500, 256, 96), (1000, 384, 128),
                                    (700, 700, 700), (1000, 1000, 1000), (1100, 1024, 1024)])
def test_ragged_sizes_padding_and_upper_untouched(hd, handle, torch_cuda, n, nb, b):
    A = oracle.spd_gram(n, 11)
    lda = n + 5
    dA, buf = padded(torch_cuda, A, lda)
    upper_marker = np.float32(-777.0)
    Au = A.copy()
    Au[np.triu_indices(n, 1)] = upper_marker
    dA, _ = padded(torch_cuda, Au, lda)
    info = info_tensor(torch_cuda)
    hd.call("double_blocked_potrf_kblocked_syrk", handle.ptr, ptr(dA), lda, n, nb, b, 37, ptr(info))
    torch_cuda.cuda.synchronize()
    handle.check()
    out = host2d(dA, lda, lda, n)
    assert int(info.item()) == 0
    assert np.all(np.isnan(out[n:, :])), "padding rows were written"
    assert np.all(out[:n][np.triu_indices(n, 1)] == upper_marker), "strict upper triangle modified"
    assert potrf_check(np.tril(out[:n]), A) <= BOUND


@pytest.mark.parametrize("fail_at", [0, 5, 64, 300, 777])
def test_not_positive_definite_info(hd, handle, torch_cuda, fail_at):
    """info = first non-positive leading minor, as LAPACK spotrf."""
    n = 1024
    A = oracle.spd_gram(n, 2).astype(np.float64)
    # make the leading minor of order fail_at+1 indefinite
    A[fail_at, fail_at] = -50.0
    A = A.astype(np.float32)
    _, linfo = oracle.lapack_spotrf(A)
    for fn in ("double_blocked_potrf", "recursive_potrf", "blocked_right_looking_potrf"):
        _, info = run_potrf(hd, handle, torch_cuda, A, fn, nb=256, b=64)
        assert info == linfo == fail_at + 1, fn


@pytest.mark.parametrize("fail_at", [0, 63, 64, 300, 1000])
@pytest.mark.parametrize("b", [512, 1024])
def test_not_positive_definite_info_block_kernel(hd, handle, torch_cuda, fail_at, b):
    """Diagonal blocks of 65..1024 are factored by one cooperative launch;
    its info must still be the first non-positive leading minor."""
    n = 1024
    A = oracle.spd_gram(n, 3).astype(np.float64)
    A[fail_at, fail_at] = -50.0
    A = A.astype(np.float32)
    _, linfo = oracle.lapack_spotrf(A)
    _, info = run_potrf(hd, handle, torch_cuda, A, "double_blocked_potrf", nb=b, b=b)
    assert info == linfo == fail_at + 1
    assert handle.device_errors() == 0


def test_zero_order_and_invalid_arguments(hd, handle, torch_cuda):
    info = info_tensor(torch_cuda)
    hd.call("double_blocked_potrf", handle.ptr, None, 1, 0, 64, 16, ptr(info))
    torch_cuda.cuda.synchronize()
    assert handle.last_status() == 0 and int(info.item()) == 0
    dA = torch_cuda.zeros(16, device="cuda")
    hd.call("double_blocked_potrf", handle.ptr, ptr(dA), 2, 4, 64, 16, ptr(info))  # lda < n
    assert handle.last_status() != 0


@pytest.mark.parametrize("n", [4096])
def test_config1_potrf_4096(hd, handle, torch_cuda, n):
    A = oracle.spd_gram(n, 0)
    L, info = run_potrf(hd, handle, torch_cuda, A, "double_blocked_potrf_kblocked_syrk",
                        nb=1024, b=256, tk=2048)
    assert info == 0
    assert oracle.scaled(oracle.potrf_residual_blas(L[:n], A), n) <= BOUND


def test_device_generator_matches_oracle(hd, handle, torch_cuda):
    x = torch_cuda.empty(100003, dtype=torch_cuda.float32, device="cuda")
    st = hd.lib().hdbf_fill_uniform(handle.ptr, ptr(x), x.numel(), 0, 17)
    torch_cuda.cuda.synchronize()
    assert st == 0
    np.testing.assert_array_equal(x.cpu().numpy(), oracle.uniform_pm1(100003, 0, offset=17))


@pytest.mark.parametrize("graphs", [True, False])
def test_graph_replay_matches_eager(hd, handle, torch_cuda, graphs):
    """The second call with identical arguments replays the recorded CUDA graph;
    results must equal the first (captured) call and the eager path bit for bit."""
    n = 1536
    A = oracle.spd_gram(n, 4)
    handle.set_graphs(graphs)
    d0 = dev(torch_cuda, A)
    d = d0.clone()
    info = info_tensor(torch_cuda)
    outs = []
    for _ in range(3):
        d.copy_(d0)
        hd.call("double_blocked_potrf_kblocked_syrk", handle.ptr, ptr(d), n, n, 512, 128, 256,
                ptr(info))
        torch_cuda.cuda.synchronize()
        handle.check()
        assert int(info.item()) == 0
        outs.append(d.cpu().numpy().copy())
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[1], outs[2])
    L = outs[2].reshape(n, n).T
    assert potrf_check(np.tril(L), A) <= BOUND
