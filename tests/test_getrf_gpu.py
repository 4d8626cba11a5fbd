"""GPU parity tests for the pivoted LU path, called through the C ABI.

Oracle: host LAPACK sgetrf (pivot sequences must be identical) and the C
restatement of the reference's CPU FP64 residual (scaled by n * eps32, bound
10); committed golden pivots in tests/golden/lapack_f32.npz."""
import os

import numpy as np
import pytest

import hygondoubleblockedfactorizations_b200 as hd_mod
import oracle
from tests.common import dev, getrf_check, host2d, info_tensor, padded, ptr

pytestmark = pytest.mark.gpu

BOUND = 10.0
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lapack_f32.npz")


def assert_pivots_match(G, ipiv, ref, what):
    """Identical pivots, or a first divergence at an FP32 near-tie (reported)."""
    pv = oracle.pivot_agreement(G, ref, ipiv)
    j = pv["first_divergence"]
    if j is not None:
        assert pv["near_tie"], f"{what}: pivots diverge: {pv}"
        print(f"{what}: first divergence at column {j}, near-tie {pv}")
    return j


def run_getrf(hd, handle, torch, A2d, fn, lda=None, outer=0, inner=0, mode=0, tblock=0,
              mtile=0, ws=None):
    n = A2d.shape[0]
    lda = lda or n
    dA, _ = padded(torch, A2d, lda)
    ipiv = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    info = info_tensor(torch)
    h = handle.ptr
    if fn == "double_blocked_getrf":
        hd.call(fn, h, ptr(dA), lda, n, outer, inner, mode, tblock, ptr(ipiv), ptr(info))
    elif fn == "double_blocked_getrf_batched_pivot":
        hd.call(fn, h, ptr(dA), lda, n, outer, inner, mode, tblock, mtile, ptr(ipiv), ptr(info),
                ws)
    elif fn == "blocked_right_looking_getrf":
        hd.call(fn, h, ptr(dA), lda, n, outer, ptr(ipiv), ptr(info))
    elif fn == "double_blocked_getrf_npvt":
        hd.call(fn, h, ptr(dA), lda, n, outer, inner, ptr(info))
    elif fn == "blocked_right_looking_getrf_npvt":
        hd.call(fn, h, ptr(dA), lda, n, outer, ptr(info))
    torch.cuda.synchronize()
    return dA, host2d(dA, lda, lda, n), ipiv.cpu().numpy()[:n], int(info.item())


def make_ws(torch, n, tile=64):
    keep = dict(src=torch.zeros(n, dtype=torch.int32, device="cuda"),
                tgt=torch.zeros(n, dtype=torch.int32, device="cuda"),
                swap=torch.zeros(n * tile, dtype=torch.float32, device="cuda"),
                hp=np.zeros(n, np.int32), hperm=np.zeros(n, np.int32),
                hs=np.zeros(n, np.int32), ht=np.zeros(n, np.int32))
    ws = hd_mod.WorkspacePivot(keep["src"].data_ptr(), keep["tgt"].data_ptr(),
                               keep["swap"].data_ptr(), keep["hp"].ctypes.data,
                               keep["hperm"].ctypes.data, keep["hs"].ctypes.data,
                               keep["ht"].ctypes.data, n, tile)
    return ws, keep


@pytest.mark.parametrize("panel", [0, 1])
@pytest.mark.parametrize("n,outer,inner", [(512, 256, 64), (1024, 512, 128), (2048, 1024, 256)])
def test_pivots_identical_to_lapack_immediate(hd, handle, torch_cuda, n, outer, inner, panel):
    # panel 0: cluster panel kernel (these blocks fit), 1: grid-wide kernel
    handle.set_panel_kernel(panel)
    G = oracle.general_uniform(n, 1)
    _, LU, ipiv, info = run_getrf(hd, handle, torch_cuda, G, "double_blocked_getrf", outer=outer,
                                  inner=inner)
    handle.check()
    assert handle.device_errors() == 0
    _, ipiv_l, info_l = oracle.lapack_sgetrf(G)
    assert info == info_l == 0
    if n <= 1024:
        np.testing.assert_array_equal(ipiv, ipiv_l)  # strict identity with this host's sgetrf
    assert_pivots_match(G, ipiv, ipiv_l, "host sgetrf")
    assert_pivots_match(G, ipiv, np.load(GOLD)[f"getrf_ipiv_{n}"], "golden sgetrf")
    assert getrf_check(LU[:n], G, ipiv) <= BOUND


@pytest.mark.parametrize("panel", [0, 1])
@pytest.mark.parametrize("mode", [0, 1])
def test_batched_pivot_variant(hd, handle, torch_cuda, mode, panel):
    import ctypes
    handle.set_panel_kernel(panel)
    n = 2048
    G = oracle.general_uniform(n, 1)
    ws, keep = make_ws(torch_cuda, n, tile=48)
    _, LU, ipiv, info = run_getrf(hd, handle, torch_cuda, G, "double_blocked_getrf_batched_pivot",
                                  outer=1024, inner=256, mode=mode, tblock=384, mtile=700,
                                  ws=ctypes.byref(ws))
    handle.check()
    assert info == 0
    assert_pivots_match(G, ipiv, np.load(GOLD)[f"getrf_ipiv_{n}"], "golden sgetrf")
    assert_pivots_match(G, ipiv, oracle.lapack_sgetrf(G)[1], "host sgetrf")
    assert getrf_check(LU[:n], G, ipiv) <= BOUND


def test_batched_pivot_invalid_workspace(hd, handle, torch_cuda):
    import ctypes
    n = 64
    G = oracle.general_uniform(n, 1)
    ws, keep = make_ws(torch_cuda, n)
    ws.capacity = n - 1
    _, _, _, info = run_getrf(hd, handle, torch_cuda, G, "double_blocked_getrf_batched_pivot",
                              outer=32, inner=16, ws=ctypes.byref(ws))
    assert info == -1 and handle.last_status() != 0


@pytest.mark.parametrize("n,outer,inner", [(1, 0, 0), (2, 1, 1), (33, 16, 8), (100, 64, 32),
                                           (257, 128, 40), (600, 300, 100), (1000, 1000, 1000)])
def test_ragged_sizes_and_padding(hd, handle, torch_cuda, n, outer, inner):
    G = oracle.general_uniform(n, 5)
    lda = n + 3
    dA, LU, ipiv, info = run_getrf(hd, handle, torch_cuda, G, "double_blocked_getrf", lda=lda,
                                   outer=outer, inner=inner)
    handle.check()
    assert info == 0
    assert np.all(np.isnan(LU[n:, :])), "padding rows written"
    _, ipiv_l, _ = oracle.lapack_sgetrf(G)
    np.testing.assert_array_equal(ipiv, ipiv_l)
    assert getrf_check(LU[:n], G, ipiv) <= BOUND


def test_right_looking_variant(hd, handle, torch_cuda):
    n = 1536
    G = oracle.general_uniform(n, 1)
    _, LU, ipiv, info = run_getrf(hd, handle, torch_cuda, G, "blocked_right_looking_getrf",
                                  outer=192)
    handle.check()
    _, ipiv_l, _ = oracle.lapack_sgetrf(G)
    np.testing.assert_array_equal(ipiv, ipiv_l)
    assert info == 0 and getrf_check(LU[:n], G, ipiv) <= BOUND


@pytest.mark.parametrize("fn", ["double_blocked_getrf_npvt", "blocked_right_looking_getrf_npvt"])
def test_no_pivot_variants(hd, handle, torch_cuda, fn):
    n = 1024
    G = oracle.general_uniform(n, 1) + np.float32(n) * np.eye(n, dtype=np.float32)
    _, LU, _, info = run_getrf(hd, handle, torch_cuda, G, fn, outer=512, inner=128)
    handle.check()
    assert info == 0
    assert getrf_check(LU[:n], G, None, pivoting=False) <= BOUND
    ref, ref_piv, _ = oracle.double_blocked_getrf(G, 512, 128)
    assert np.array_equal(ref_piv, np.arange(1, n + 1))  # diagonal dominance: no row swaps
    assert np.abs(LU[:n] - ref).max() <= 1e-4 * np.abs(ref).max()


def test_singular_info(hd, handle, torch_cuda):
    """Exact zero pivot: info = first zero U(i,i) (LAPACK sgetrf)."""
    n = 300
    G = oracle.general_uniform(n, 9)
    G[:, 77] = 0.0
    _, LU, ipiv, info = run_getrf(hd, handle, torch_cuda, G, "double_blocked_getrf", outer=128,
                                  inner=32)
    _, ipiv_l, info_l = oracle.lapack_sgetrf(G)
    assert info == info_l == 78
    np.testing.assert_array_equal(ipiv[:77], ipiv_l[:77])


def test_apply_panel_pivots_launcher(hd, handle, torch_cuda):
    """launch_apply_getrf_panel_pivots vs the reference kernel's semantics."""
    n, panel, size = 300, 40, 50
    rng = np.random.default_rng(0)
    A = rng.standard_normal((n, n)).astype(np.float32)
    piv = np.array([rng.integers(o + 1, n - panel + 1) for o in range(size)], dtype=np.int32)
    want = A.copy()
    for c in range(n):
        if panel <= c < panel + size:
            continue
        for o in range(size):
            r, pr = panel + o, panel + piv[o] - 1
            want[[r, pr], c] = want[[pr, r], c]
    dA = dev(torch_cuda, A)
    dp = dev(torch_cuda, piv)
    stream = torch_cuda.cuda.current_stream().cuda_stream
    hd.call("launch_apply_getrf_panel_pivots", ptr(dA), n, n, panel, size, ptr(dp), stream)
    torch_cuda.cuda.synchronize()
    np.testing.assert_array_equal(host2d(dA, n, n, n), want)
    np.testing.assert_array_equal(dp.cpu().numpy(), piv + panel)


def test_apply_permutation_launcher(hd, handle, torch_cuda):
    n, cols, tile = 400, 37, 8
    rng = np.random.default_rng(1)
    A = rng.standard_normal((n, cols)).astype(np.float32)
    rows = rng.choice(n, 60, replace=False).astype(np.int32)
    src = rows.copy()
    tgt = rng.permutation(rows).astype(np.int32)
    want = A.copy()
    want[tgt, :] = A[src, :]
    dA = dev(torch_cuda, A)
    ds, dt = dev(torch_cuda, src), dev(torch_cuda, tgt)
    tmp = torch_cuda.zeros(60 * tile, dtype=torch_cuda.float32, device="cuda")
    stream = torch_cuda.cuda.current_stream().cuda_stream
    hd.call("launch_apply_getrf_permutation", ptr(dA), n, cols, ptr(ds), ptr(dt), 60, ptr(tmp),
            tile, stream)
    torch_cuda.cuda.synchronize()
    np.testing.assert_array_equal(host2d(dA, n, n, cols), want)


def test_graph_replay_getrf(hd, handle, torch_cuda):
    """Replaying the recorded LU graph reproduces the captured run exactly."""
    n = 1024
    G = oracle.general_uniform(n, 1)
    d0 = dev(torch_cuda, G)
    d = d0.clone()
    ipiv = torch_cuda.zeros(n, dtype=torch_cuda.int32, device="cuda")
    info = info_tensor(torch_cuda)
    outs = []
    for _ in range(3):
        d.copy_(d0)
        hd.call("double_blocked_getrf", handle.ptr, ptr(d), n, n, 512, 128, 1, 256, ptr(ipiv),
                ptr(info))
        torch_cuda.cuda.synchronize()
        handle.check()
        outs.append((d.cpu().numpy().copy(), ipiv.cpu().numpy().copy(), int(info.item())))
    for o in outs[1:]:
        np.testing.assert_array_equal(o[0], outs[0][0])
        np.testing.assert_array_equal(o[1], outs[0][1])
        assert o[2] == 0
    np.testing.assert_array_equal(outs[0][1], oracle.lapack_sgetrf(G)[1])


def test_panel_kernels_agree_bitwise_large(hd, handle, torch_cuda):
    """n = 16384 with 32-column leaves: the first panels run on 16-CTA clusters,
    later ones on 8, 4, 2 and 1; the grid-wide kernel must give bit-identical
    factors and pivots (same arithmetic, same order).  Pivots follow host sgetrf up to FP32
    near-ties; the residual is the FP64 ||PA - LU||_F / ||A||_F (GPU FP64,
    same formula as the oracle), scaled by n * eps32."""
    import os
    n = 16384
    G = oracle.general_uniform(n, 1)
    out = {}
    os.environ["HDBF_PANEL_LEAF"] = "32"  # same recursion for both kernels
    try:
        h32 = hd.Handle(torch_cuda.cuda.current_stream().cuda_stream)
    finally:
        del os.environ["HDBF_PANEL_LEAF"]
    for panel in (2, 1):  # 2: cluster kernel, 1: grid-wide kernel
        h32.set_panel_kernel(panel)
        dA, _, ipiv, info = run_getrf(hd, h32, torch_cuda, G, "double_blocked_getrf",
                                      outer=4096, inner=512)
        assert info == 0 and h32.device_errors() == 0
        out[panel] = (dA.clone(), ipiv)
    h32.close()
    out[0] = out[2]
    # the default (128-column leaves) must also follow host sgetrf
    _, _, ipiv128, info = run_getrf(hd, handle, torch_cuda, G, "double_blocked_getrf",
                                    outer=4096, inner=512)
    assert info == 0
    lapack_piv = oracle.lapack_sgetrf(G)[1]
    assert_pivots_match(G, ipiv128, lapack_piv, "host sgetrf (leaf 128)")
    assert np.array_equal(out[0][1], out[1][1])
    assert torch_cuda.equal(out[0][0], out[1][0])
    ipiv = out[0][1]
    assert_pivots_match(G, ipiv, lapack_piv, "host sgetrf")
    torch = torch_cuda
    LU = out[0][0].view(n, n).t().double()  # row-major view of the column-major factor
    L = torch.tril(LU, -1) + torch.eye(n, dtype=torch.float64, device="cuda")
    U = torch.triu(LU)
    A = torch.from_numpy(np.ascontiguousarray(G)).cuda().double()
    perm = np.arange(n)
    for i, p in enumerate(ipiv - 1):
        perm[i], perm[p] = perm[p], perm[i]
    PA = A[torch.from_numpy(perm).cuda()]
    r = (torch.linalg.matrix_norm(PA - L @ U) / torch.linalg.matrix_norm(A)).item()
    assert r / (n * 2.0 ** -23) <= BOUND, r


@pytest.mark.parametrize("n,outer,inner,mode,tblock,mtile", [
    (3072, 1024, 256, 0, 0, 0),      # three outer blocks, four chunks each
    (2500, 768, 128, 1, 384, 500),   # ragged last block, iterative outer TRSM
    (4096, 2048, 32, 0, 0, 0),       # 64 inner panels per block: chunks of two panels
])
def test_lookahead_bitwise_batched(hd, handle, torch_cuda, n, outer, inner, mode, tblock, mtile):
    """Look-ahead (panel chain on the internal stream, outer GEMM in chunks,
    running composed interchanges) moves the same data and runs the same
    arithmetic as the serial schedule: factors and pivots are bit-identical,
    graph capture included (the second call of each replays its graph)."""
    import ctypes
    G = oracle.general_uniform(n, 3)
    ws, keep = make_ws(torch_cuda, n, tile=64)
    out = {}
    try:
        for la in (0, 1):
            handle.set_lookahead(la)
            for rep in range(2):
                dA, LU, ipiv, info = run_getrf(hd, handle, torch_cuda, G,
                                               "double_blocked_getrf_batched_pivot", outer=outer,
                                               inner=inner, mode=mode, tblock=tblock, mtile=mtile,
                                               ws=ctypes.byref(ws))
                handle.check()
                assert info == 0 and handle.device_errors() == 0
                out[(la, rep)] = (dA.clone(), ipiv)
    finally:
        handle.set_lookahead(1)
    for k in out:
        assert torch_cuda.equal(out[k][0], out[(0, 0)][0]), k
        np.testing.assert_array_equal(out[k][1], out[(0, 0)][1])
    assert_pivots_match(G, out[(1, 0)][1], oracle.lapack_sgetrf(G)[1], "host sgetrf")
    LU = host2d(out[(1, 0)][0], n, n, n)
    assert getrf_check(LU[:n], G, out[(1, 0)][1]) <= BOUND


def test_lookahead_npvt_and_ragged(hd, handle, torch_cuda):
    """No-pivot look-ahead is bit-identical to the serial schedule; a last
    outer block narrower than 32 columns (the serial path may take the
    split-K skinny GEMM there) still factors to the residual bound."""
    import ctypes
    n = 2048
    G = oracle.general_uniform(n, 5) + np.float32(n) * np.eye(n, dtype=np.float32)
    res = {}
    try:
        for la in (0, 1):
            handle.set_lookahead(la)
            dA, LU, _, info = run_getrf(hd, handle, torch_cuda, G, "double_blocked_getrf_npvt",
                                        outer=512, inner=128)
            handle.check()
            assert info == 0
            res[la] = dA.clone()
        assert torch_cuda.equal(res[0], res[1])
        assert getrf_check(host2d(res[1], n, n, n)[:n], G, None, pivoting=False) <= BOUND
        n2 = 1024 + 20
        G2 = oracle.general_uniform(n2, 6)
        ws, keep = make_ws(torch_cuda, n2)
        handle.set_lookahead(1)
        _, LU2, ipiv2, info2 = run_getrf(hd, handle, torch_cuda, G2,
                                         "double_blocked_getrf_batched_pivot", outer=512,
                                         inner=128, ws=ctypes.byref(ws))
        handle.check()
        assert info2 == 0
        assert_pivots_match(G2, ipiv2, oracle.lapack_sgetrf(G2)[1], "host sgetrf")
        assert getrf_check(LU2[:n2], G2, ipiv2) <= BOUND
    finally:
        handle.set_lookahead(1)


def test_panel_exchange_after_narrow_launch(hd, handle, torch_cuda):
    """Grid-wide panel launches of 65..67 columns followed by further launches
    (the exchange words of one launch must never be taken for the next's):
    pivots follow host sgetrf and the factors meet the residual bound."""
    handle.set_panel_kernel(1)
    try:
        for n, nb in ((1090, 1024), (2115, 1024), (3000, 67)):
            G = oracle.general_uniform(n, 11)
            _, LU, ipiv, info = run_getrf(hd, handle, torch_cuda, G,
                                          "blocked_right_looking_getrf", outer=nb)
            handle.check()
            assert info == 0 and handle.device_errors() == 0
            assert_pivots_match(G, ipiv, oracle.lapack_sgetrf(G)[1], "host sgetrf")
            assert getrf_check(LU[:n], G, ipiv) <= BOUND
    finally:
        handle.set_panel_kernel(0)


@pytest.mark.parametrize("fn", ["double_blocked_getrf", "double_blocked_getrf_batched_pivot"])
def test_long_swap_sequences(hd, handle, torch_cuda, fn):
    """Inner panels of 4608 columns: their swap sequences are longer than the
    sorted-group composition takes (4096), so the one-thread replay composes
    them; inside the panel the recursion's halves use the sorted-group
    kernel.  Pivots follow host sgetrf; residual within the bound."""
    import ctypes
    n = 4608 + 77
    G = oracle.general_uniform(n, 13)
    kw = {}
    if fn.endswith("batched_pivot"):
        ws, keep = make_ws(torch_cuda, n, tile=32)
        kw = dict(ws=ctypes.byref(ws))
    _, LU, ipiv, info = run_getrf(hd, handle, torch_cuda, G, fn, outer=4608, inner=4608, **kw)
    handle.check()
    assert info == 0 and handle.device_errors() == 0
    assert_pivots_match(G, ipiv, oracle.lapack_sgetrf(G)[1], "host sgetrf")
    assert oracle.scaled(oracle.getrf_residual_tiled(LU[:n], G, ipiv), n) <= BOUND
