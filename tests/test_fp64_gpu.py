"""GPU parity tests for the FP64 twins (the reference's `_double` entry
points), called through the C ABI.

Oracle: host LAPACK dpotrf / dgetrf (SciPy OpenBLAS) for factors, info and
pivot sequences, and the FP64 residuals ||A - L L^T||_F / ||A||_F and
||P A - L U||_F / ||A||_F scaled by n * eps64 (eps64 = 2^-52, bound 10).
Pivot sequences must equal LAPACK's up to a near-tie at FP64 rounding level
(relative gap of the two largest candidates below 1e-10)."""
import ctypes

import numpy as np
import pytest

import hygondoubleblockedfactorizations_b200 as hd_mod
import oracle
from tests.common import dev, host2d, info_tensor, padded, ptr

pytestmark = pytest.mark.gpu

EPS64 = 2.0 ** -52
BOUND = 10.0
NEAR_TIE64 = 1e-10


def spd64(n, seed):
    G = oracle.general_uniform(n, seed).astype(np.float64)
    A = G @ G.T / max(n, 1) + np.eye(n)
    return 0.5 * (A + A.T)


def gen64(n, seed):
    return oracle.general_uniform(n, seed).astype(np.float64)


def chol_resid(L, A):
    n = A.shape[0]
    Lt = np.tril(L)
    return np.linalg.norm(A - Lt @ Lt.T) / np.linalg.norm(A) / (n * EPS64)


def lu_resid(LU, A, ipiv):
    n = A.shape[0]
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    PA = A.copy()
    if ipiv is not None:
        for i, p in enumerate(ipiv):
            p = int(p) - 1
            if p != i:
                PA[[i, p], :] = PA[[p, i], :]
    return np.linalg.norm(PA - L @ U) / np.linalg.norm(A) / (n * EPS64)


def assert_pivots64(A, ipiv, ref):
    pv = oracle.pivot_agreement(A, ref, ipiv, unit_roundoff=2.0 ** -53, rel_tie=NEAR_TIE64)
    assert pv["near_tie"], f"pivots diverge: {pv}"


POTRF_CASES = [
    ("double_blocked_potrf_double", (256, 64)),
    ("double_blocked_potrf_double_dbtrsm", (256, 128)),
    ("double_blocked_potrf_double_kblocked_syrk", (256, 64, 200)),
    ("double_blocked_potrf_double_kblocked_syrk_adaptive_gemm", (512, 128, 0)),
    ("double_blocked_potrf_double_kblocked_syrk_adaptive_gemm_configured",
     (256, 64, 300, 100, 50, 64)),
    ("blocked_right_looking_potrf_double", (192,)),
    ("recursive_potrf_double", (100,)),
]


def run_potrf64(hd, handle, torch, fn, A, params, lda):
    n = A.shape[0]
    dA, _ = padded(torch, A, lda, dtype=np.float64)
    info = info_tensor(torch)
    h = handle.ptr
    if fn == "blocked_right_looking_potrf_double":
        hd.call(fn, h, ptr(dA), lda, n, params[0], ptr(info))
    elif fn == "recursive_potrf_double":
        hd.call(fn, h, None, ptr(dA), lda, n, params[0], ptr(info))
    else:
        hd.call(fn, h, ptr(dA), lda, n, *params, ptr(info))
    torch.cuda.synchronize()
    return dA, host2d(dA, lda, lda, n), int(info.item())


@pytest.mark.parametrize("fn,params", POTRF_CASES)
@pytest.mark.parametrize("n,pad", [(1, 0), (64, 0), (65, 3), (700, 1), (1500, 0)])
def test_potrf_double_variants(hd, handle, torch_cuda, fn, params, n, pad):
    A = spd64(n, 2)
    lda = n + pad
    dA, L, info = run_potrf64(hd, handle, torch_cuda, fn, A, params, lda)
    handle.check()
    assert info == 0 and handle.device_errors() == 0
    from scipy.linalg import lapack
    ref, rinfo = lapack.dpotrf(np.asfortranarray(A), lower=1, clean=1)
    assert rinfo == 0
    Ln = np.tril(L[:n])
    assert np.abs(Ln - ref).max() <= 1e-11 * np.abs(ref).max()
    assert chol_resid(L[:n], A) <= BOUND
    iu = np.triu_indices(n, 1)
    np.testing.assert_array_equal(L[:n][iu], A[iu])  # strict upper triangle untouched
    if pad:
        assert np.all(np.isnan(L[n:]))


@pytest.mark.parametrize("k", [0, 63, 64, 300, 899])
def test_potrf_double_info(hd, handle, torch_cuda, k):
    n = 900
    A = spd64(n, 4)
    A[k, k] = -1.0
    from scipy.linalg import lapack
    _, rinfo = lapack.dpotrf(np.asfortranarray(A), lower=1)
    for fn, params in (("double_blocked_potrf_double", (256, 64)),
                       ("blocked_right_looking_potrf_double", (128,))):
        _, _, info = run_potrf64(hd, handle, torch_cuda, fn, A, params, n)
        assert info == rinfo == k + 1, (fn, info, rinfo)


def make_ws64(torch, n, tile=16):
    keep = dict(src=torch.zeros(n, dtype=torch.int32, device="cuda"),
                tgt=torch.zeros(n, dtype=torch.int32, device="cuda"),
                swap=torch.zeros(n * tile, dtype=torch.float64, device="cuda"),
                hp=np.zeros(n, np.int32), hperm=np.zeros(n, np.int32),
                hs=np.zeros(n, np.int32), ht=np.zeros(n, np.int32))
    ws = hd_mod.WorkspacePivot(keep["src"].data_ptr(), keep["tgt"].data_ptr(),
                               keep["swap"].data_ptr(), keep["hp"].ctypes.data,
                               keep["hperm"].ctypes.data, keep["hs"].ctypes.data,
                               keep["ht"].ctypes.data, n, tile)
    return ws, keep


def run_getrf64(hd, handle, torch, fn, A, lda, outer=0, inner=0, mode=0, tblock=0, mtile=0):
    n = A.shape[0]
    dA, _ = padded(torch, A, lda, dtype=np.float64)
    ipiv = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    info = info_tensor(torch)
    h = handle.ptr
    keep = None
    if fn == "double_blocked_getrf_double":
        hd.call(fn, h, ptr(dA), lda, n, outer, inner, mode, tblock, ptr(ipiv), ptr(info))
    elif fn == "double_blocked_getrf_double_batched_pivot":
        ws, keep = make_ws64(torch, n)
        hd.call(fn, h, ptr(dA), lda, n, outer, inner, mode, tblock, mtile, ptr(ipiv), ptr(info),
                ctypes.byref(ws))
    elif fn == "blocked_right_looking_getrf_double":
        hd.call(fn, h, ptr(dA), lda, n, outer, ptr(ipiv), ptr(info))
    elif fn == "double_blocked_getrf_npvt_double":
        hd.call(fn, h, ptr(dA), lda, n, outer, inner, ptr(info))
    elif fn == "blocked_right_looking_getrf_npvt_double":
        hd.call(fn, h, ptr(dA), lda, n, outer, ptr(info))
    torch.cuda.synchronize()
    del keep
    return dA, host2d(dA, lda, lda, n), ipiv.cpu().numpy()[:n], int(info.item())


GETRF_CASES = [
    ("double_blocked_getrf_double", dict(outer=512, inner=128, mode=0)),
    ("double_blocked_getrf_double", dict(outer=512, inner=96, mode=1, tblock=192)),
    ("double_blocked_getrf_double_batched_pivot", dict(outer=512, inner=128, mode=1, tblock=256,
                                                       mtile=300)),
    ("blocked_right_looking_getrf_double", dict(outer=200)),
]


@pytest.mark.parametrize("fn,kw", GETRF_CASES)
@pytest.mark.parametrize("n,pad", [(1, 0), (64, 0), (65, 2), (1000, 1), (2051, 0)])
def test_getrf_double_variants(hd, handle, torch_cuda, fn, kw, n, pad):
    A = gen64(n, 7)
    lda = n + pad
    dA, LU, ipiv, info = run_getrf64(hd, handle, torch_cuda, fn, A, lda, **kw)
    handle.check()
    assert info == 0 and handle.device_errors() == 0
    ref_lu, ref_piv, rinfo = oracle.lapack_dgetrf(A)
    assert rinfo == 0
    assert_pivots64(A, ipiv, ref_piv)
    if np.array_equal(ipiv, ref_piv):
        assert np.abs(LU[:n] - ref_lu).max() <= 1e-10 * np.abs(ref_lu).max()
    assert lu_resid(LU[:n], A, ipiv) <= BOUND
    if pad:
        assert np.all(np.isnan(LU[n:]))


@pytest.mark.parametrize("fn", ["double_blocked_getrf_npvt_double",
                                "blocked_right_looking_getrf_npvt_double"])
def test_getrf_double_npvt(hd, handle, torch_cuda, fn):
    n = 1100
    A = gen64(n, 8) + n * np.eye(n)
    _, LU, _, info = run_getrf64(hd, handle, torch_cuda, fn, A, n, outer=256, inner=64)
    handle.check()
    assert info == 0
    assert lu_resid(LU[:n], A, None) <= BOUND


@pytest.mark.parametrize("zero_col", [0, 70, 555])
def test_getrf_double_singular_info(hd, handle, torch_cuda, zero_col):
    n = 600
    A = gen64(n, 9)
    A[:, zero_col] = 0.0
    _, _, rinfo = oracle.lapack_dgetrf(A)
    for fn, kw in (("double_blocked_getrf_double", dict(outer=256, inner=64)),
                   ("blocked_right_looking_getrf_double", dict(outer=128))):
        _, _, _, info = run_getrf64(hd, handle, torch_cuda, fn, A, n, **kw)
        assert info == rinfo == zero_col + 1, (fn, info, rinfo)


def test_getrf_double_graph_replay(hd, handle, torch_cuda):
    """Three calls on the same buffers: the first records the CUDA graph, the
    next two replay it; all three give bit-identical factors and pivots."""
    n = 1024
    A = gen64(n, 10)
    d0 = dev(torch_cuda, A)
    d = d0.clone()
    ipiv = torch_cuda.zeros(n, dtype=torch_cuda.int32, device="cuda")
    info = info_tensor(torch_cuda)
    outs = []
    for _ in range(3):
        d.copy_(d0)
        hd.call("double_blocked_getrf_double", handle.ptr, ptr(d), n, n, 512, 128, 1, 256,
                ptr(ipiv), ptr(info))
        torch_cuda.cuda.synchronize()
        handle.check()
        assert int(info.item()) == 0
        outs.append((d.clone(), ipiv.cpu().numpy().copy()))
    for o in outs[1:]:
        assert torch_cuda.equal(o[0], outs[0][0])
        np.testing.assert_array_equal(o[1], outs[0][1])
    assert_pivots64(A, outs[0][1], oracle.lapack_dgetrf(A)[1])


def test_blas_double_twins(hd, handle, torch_cuda):
    rng = np.random.default_rng(11)
    h = handle.ptr
    n, k, rows = 300, 170, 250
    A = rng.standard_normal((n, k))
    C0 = rng.standard_normal((n, n))
    want = C0 - A @ A.T
    for fn, extra in (("syrk_lower_update_double", ()),
                      ("syrk_lower_update_kblocked_double", (64,))):
        dA, dC = dev(torch_cuda, A), dev(torch_cuda, C0)
        hd.call(fn, h, n, k, ptr(dA), n, ptr(dC), n, *extra)
        torch_cuda.cuda.synchronize()
        C = host2d(dC, n, n, n)
        il = np.tril_indices(n)
        assert np.abs(C[il] - want[il]).max() <= 1e-12 * np.abs(want).max(), fn
        iu = np.triu_indices(n, 1)
        np.testing.assert_array_equal(C[iu], C0[iu])
    for fn in ("recursive_syrk_parallel_double", "batched_syrk_bottom_up_double"):
        dA, dC = dev(torch_cuda, A), dev(torch_cuda, C0)
        if fn == "recursive_syrk_parallel_double":
            hd.call(fn, h, ptr(dA), n, ptr(dC), n, n, k, 64)
        else:
            hd.call(fn, h, None, ptr(dA), n, ptr(dC), n, n, k, 64)
        torch_cuda.cuda.synchronize()
        C = host2d(dC, n, n, n)
        il = np.tril_indices(n)
        assert np.abs(C[il] - want[il]).max() <= 1e-12 * np.abs(want).max(), fn
    # C -= A B^T (plain and M-tiled)
    B = rng.standard_normal((n - 20, k))
    C1 = rng.standard_normal((rows, n - 20))
    want = C1 - A[:rows] @ B.T
    for fn, extra in (("gemm_nt_update_double", ()), ("gemm_nt_update_m_tiled_double", (96,))):
        dA, dB, dC = dev(torch_cuda, A), dev(torch_cuda, B), dev(torch_cuda, C1)
        hd.call(fn, h, rows, n - 20, k, ptr(dA), n, ptr(dB), n - 20, ptr(dC), rows, *extra)
        torch_cuda.cuda.synchronize()
        assert np.abs(host2d(dC, rows, rows, n - 20) - want).max() <= 1e-12 * np.abs(want).max()
    # B <- B L^{-T}: one-shot, double-blocked and recursive
    m = 333
    L = np.linalg.cholesky(spd64(m, 12))
    Bt = rng.standard_normal((rows, m))
    want = np.linalg.solve(L, Bt.T).T
    for fn, extra in (("trsm_right_lower_transpose_double", None),
                      ("double_blocked_trsm_double", (128, 64)),
                      ("recursive_trsm_double", (100,))):
        dL, dB = dev(torch_cuda, L), dev(torch_cuda, Bt)
        if extra is None:
            hd.call(fn, h, rows, m, ptr(dL), m, ptr(dB), rows)
        else:
            hd.call(fn, h, ptr(dL), m, ptr(dB), rows, rows, m, *extra)
        torch_cuda.cuda.synchronize()
        handle.check()
        got = host2d(dB, rows, rows, m)
        assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max(), fn


def test_pivot_launchers_double(hd, handle, torch_cuda):
    n, panel, size = 300, 40, 50
    rng = np.random.default_rng(13)
    A = rng.standard_normal((n, n))
    piv = np.array([rng.integers(o + 1, n - panel + 1) for o in range(size)], dtype=np.int32)
    want = A.copy()
    for c in range(n):
        if panel <= c < panel + size:
            continue
        for o in range(size):
            r, pr = panel + o, panel + piv[o] - 1
            want[[r, pr], c] = want[[pr, r], c]
    dA, dp = dev(torch_cuda, A), dev(torch_cuda, piv)
    stream = torch_cuda.cuda.current_stream().cuda_stream
    hd.call("launch_apply_getrf_panel_pivots_double", ptr(dA), n, n, panel, size, ptr(dp),
            stream)
    torch_cuda.cuda.synchronize()
    np.testing.assert_array_equal(host2d(dA, n, n, n), want)
    np.testing.assert_array_equal(dp.cpu().numpy(), piv + panel)

    cols, tile = 37, 8
    A = rng.standard_normal((400, cols))
    rows = rng.choice(400, 60, replace=False).astype(np.int32)
    src, tgt = rows.copy(), rng.permutation(rows).astype(np.int32)
    want = A.copy()
    want[tgt, :] = A[src, :]
    dA, ds, dt = dev(torch_cuda, A), dev(torch_cuda, src), dev(torch_cuda, tgt)
    tmp = torch_cuda.zeros(60 * tile, dtype=torch_cuda.float64, device="cuda")
    hd.call("launch_apply_getrf_permutation_double", ptr(dA), 400, cols, ptr(ds), ptr(dt), 60,
            ptr(tmp), tile, stream)
    torch_cuda.cuda.synchronize()
    np.testing.assert_array_equal(host2d(dA, 400, 400, cols), want)
