"""GPU test of trsm_right_lower_transpose_noalloc, the allocation-free variant
of trsm_right_lower_transpose for callers that cannot allocate device memory
(services whose device memory is fixed at start-up, libraries that may only
use caller-owned buffers).  It keeps its scratch in a fixed device array
inside the library, so this file is collected last: a failure here cannot
hide the result of any other test."""
import numpy as np
import pytest

from tests.common import dev, host2d, ptr

pytestmark = pytest.mark.gpu

MAX_COLS = 4096  # HDBF_NOALLOC_TRSM_MAX_COLS


def lower_factor(m, seed):
    rng = np.random.default_rng(seed)
    L = np.tril(rng.uniform(-1, 1, size=(m, m))) * 0.1
    L[np.diag_indices(m)] = 1.0 + np.abs(rng.uniform(-1, 1, size=m))
    return L.astype(np.float32)


def rel_err(got, want):
    return np.abs(got.astype(np.float64) - want).max() / max(1e-30, np.abs(want).max())


@pytest.mark.parametrize("rows,cols", [(1000, 300), (4096, 1024), (512, MAX_COLS)])
def test_noalloc_matches_regular_entry_point_twice(hd, handle, torch_cuda, rows, cols):
    L = lower_factor(cols, 7)
    B = np.random.default_rng(8).uniform(-1, 1, size=(rows, cols)).astype(np.float32)
    dL = dev(torch_cuda, L)
    ref = dev(torch_cuda, B)
    hd.call("trsm_right_lower_transpose", handle.ptr, rows, cols, ptr(dL), cols, ptr(ref), rows)
    torch_cuda.cuda.synchronize()
    handle.check("trsm_right_lower_transpose")
    want = host2d(ref, rows, rows, cols)
    stream = torch_cuda.cuda.current_stream().cuda_stream
    for call in range(2):  # the shared scratch keeps the previous call's contents
        d = dev(torch_cuda, B)
        st = hd.call("trsm_right_lower_transpose_noalloc", rows, cols, ptr(dL), cols, ptr(d), rows,
                     stream)
        torch_cuda.cuda.synchronize()
        assert st == 0, f"call {call}: status {st}"
        got = host2d(d, rows, rows, cols)
        assert rel_err(got, want) <= 1e-4, f"call {call}"
    exact = np.linalg.solve(L.astype(np.float64), B.astype(np.float64).T).T
    assert rel_err(got, exact) <= 1e-4


def test_noalloc_rejects_too_many_columns(hd, torch_cuda):
    rows, cols = 8, MAX_COLS + 1
    dL = torch_cuda.zeros(cols * cols // 64, dtype=torch_cuda.float32, device="cuda")
    d = torch_cuda.full((rows * cols,), 3.0, dtype=torch_cuda.float32, device="cuda")
    stream = torch_cuda.cuda.current_stream().cuda_stream
    st = hd.call("trsm_right_lower_transpose_noalloc", rows, cols, ptr(dL), cols, ptr(d), rows,
                 stream)
    torch_cuda.cuda.synchronize()
    assert st != 0
    assert bool((d == 3.0).all())
