"""FP32 GEMM code paths, through the C ABI against an FP64 product:
interior tiles (no bounds tests) next to ragged edge tiles, and the split-K
path that under-filled launches take (fewer tiles than SMs: K cut into
chunks whose partial products are summed in chunk order; it needs the
handle's workspace, reserved first), for the plain update (gemm_nt_update)
and the lower-triangular one (syrk_lower_update)."""
import ctypes

import pytest

from tests.common import ptr

pytestmark = pytest.mark.gpu


def uniform(torch, hd, handle, count, seed):
    x = torch.empty(count, dtype=torch.float32, device="cuda")
    assert hd.lib().hdbf_fill_uniform(handle.ptr, ctypes.c_void_p(x.data_ptr()), count, seed, 0) == 0
    return x


@pytest.mark.parametrize("M,N,K", [
    (4096, 2048, 1024),   # interior tiles only, full waves
    (4000, 1000, 1000),   # ragged edges, K not a multiple of the K step
    (1024, 512, 4096),    # 32 tiles: split K
    (1000, 300, 4100),    # split K with ragged tiles and a short last chunk
])
def test_gemm_nt_update_paths(hd, handle, torch_cuda, M, N, K):
    torch = torch_cuda
    handle.reserve(hd.lib().hdbf_workspace_bytes_for(64))
    A = uniform(torch, hd, handle, M * K, 1)
    B = uniform(torch, hd, handle, N * K, 2)
    C = uniform(torch, hd, handle, M * N, 3)
    want = (C.view(N, M).t().double()
            - A.view(K, M).t().double() @ B.view(K, N).t().double().t())
    hd.call("gemm_nt_update", handle.ptr, M, N, K, ptr(A), M, ptr(B), N, ptr(C), M)
    torch.cuda.synchronize()
    handle.check()
    got = C.view(N, M).t().double()
    err = float((got - want).abs().max() / want.abs().max())
    assert err <= 2e-6 * (K / 1000) ** 0.5 * 4, err


@pytest.mark.parametrize("n,k", [(2048, 1024), (640, 4096), (1000, 3000)])
def test_syrk_lower_update_paths(hd, handle, torch_cuda, n, k):
    torch = torch_cuda
    handle.reserve(hd.lib().hdbf_workspace_bytes_for(64))
    A = uniform(torch, hd, handle, n * k, 4)
    C = uniform(torch, hd, handle, n * n, 5)
    C0 = C.view(n, n).t().double().clone()
    Am = A.view(k, n).t().double()
    want = torch.tril(C0 - Am @ Am.t()) + torch.triu(C0, 1)  # upper triangle untouched
    hd.call("syrk_lower_update", handle.ptr, n, k, ptr(A), n, ptr(C), n)
    torch.cuda.synchronize()
    handle.check()
    got = C.view(n, n).t().double()
    assert torch.equal(torch.triu(got, 1), torch.triu(C0, 1))
    err = float((got - want).abs().max() / want.abs().max())
    assert err <= 2e-6 * (k / 1000) ** 0.5 * 4, err
