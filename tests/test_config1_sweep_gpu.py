"""Config-1 parity at the sweep's smaller orders, through the C ABI.

POTRF (double_blocked_potrf_kblocked_syrk) on A = G G^T / n + I and pivoted
GETRF (double_blocked_getrf_batched_pivot, iterative outer TRSM) on U[-1,1)
with the bench's blocks clamped to n.  Checked like the reference's verify
step after a timed run (potrf_benchmark_common.cpp:294-344,
getrf_benchmark_common.cpp:54-72): the CPU FP64 scaled residual (block-column
oracle, pinned to the C restatement by the CPU tests) <= 10, and the GPU pivot
sequence against host LAPACK sgetrf's -- identical, or a first divergence at an
FP32 near-tie.  Orders 32768 and 49152 run in ``bench.py --sweep`` (minutes
of host LAPACK and FP64 residual work per order)."""
import ctypes

import numpy as np
import pytest

import oracle
from tests.common import ptr
from tests.test_getrf_gpu import make_ws

pytestmark = pytest.mark.gpu

BOUND = 10.0
POTRF_BLOCKS = (4096, 512)
GETRF_BLOCKS = (8192, 1024)


def spd_on_device(torch, n):
    """G G^T / n + I formed in FP64 on the device, rounded to FP32 (G iid
    U[-1,1), seed 0); returns (device flat column-major, host 2-D)."""
    G = torch.from_numpy(np.ascontiguousarray(oracle.general_uniform(n, 0).T)).cuda().double()
    A = (G.t() @ G).div_(n)  # G holds the transpose: G.t() @ G = G0 G0^T
    A = 0.5 * (A + A.t())
    A.diagonal().add_(1.0)
    A32 = A.float().contiguous()  # symmetric: row-major storage = column-major storage
    del A, G
    return A32.reshape(-1), A32.cpu().numpy()


@pytest.mark.parametrize("n", [4096, 8192, 16384])
def test_config1_potrf(hd, handle, torch_cuda, n):
    torch = torch_cuda
    dA, A = spd_on_device(torch, n)
    info = torch.full((1,), 12345, dtype=torch.int32, device="cuda")
    nb, b = min(n, POTRF_BLOCKS[0]), POTRF_BLOCKS[1]
    hd.call("double_blocked_potrf_kblocked_syrk", handle.ptr, ptr(dA), n, n, nb, b, 0, ptr(info))
    torch.cuda.synchronize()
    handle.check()
    assert int(info.item()) == 0 and handle.device_errors() == 0
    L = dA.cpu().numpy().reshape(n, n).T
    r = oracle.scaled(oracle.potrf_residual_tiled(L, A), n)
    assert r <= BOUND, r
    Lh, info_h = oracle.lapack_spotrf(A)
    assert info_h == 0
    rh = oracle.scaled(oracle.potrf_residual_tiled(Lh, A), n)
    print(f"n={n}: POTRF scaled residual {r:.3g} (host spotrf {rh:.3g})")


@pytest.mark.parametrize("n", [4096, 8192, 16384])
def test_config1_getrf(hd, handle, torch_cuda, n):
    torch = torch_cuda
    G = oracle.general_uniform(n, 1)
    dG = torch.empty(n * n, dtype=torch.float32, device="cuda")
    assert hd.lib().hdbf_fill_uniform(handle.ptr, ctypes.c_void_p(dG.data_ptr()), n * n, 1, 0) == 0
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.full((1,), 12345, dtype=torch.int32, device="cuda")
    ws, keep = make_ws(torch, n, tile=64)
    nb, b = min(n, GETRF_BLOCKS[0]), GETRF_BLOCKS[1]
    hd.call("double_blocked_getrf_batched_pivot", handle.ptr, ptr(dG), n, n, nb, b, 1, 0, 0,
            ptr(ipiv), ptr(info), ctypes.byref(ws))
    torch.cuda.synchronize()
    handle.check()
    assert int(info.item()) == 0 and handle.device_errors() == 0
    LU = dG.cpu().numpy().reshape(n, n).T
    piv = ipiv.cpu().numpy()
    r = oracle.scaled(oracle.getrf_residual_tiled(LU, G, piv), n)
    assert r <= BOUND, r
    _, piv_h, info_h = oracle.lapack_sgetrf(G)
    assert info_h == 0
    pv = oracle.pivot_agreement(G, piv_h, piv)
    assert pv["near_tie"], f"pivots diverge: {pv}"
    print(f"n={n}: GETRF scaled residual {r:.3g}; pivots vs sgetrf: "
          + ("identical" if pv["first_divergence"] is None else f"near-tie divergence {pv}"))
