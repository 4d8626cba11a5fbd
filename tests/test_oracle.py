"""CPU tests of the oracle: the C restatement of the reference's FP64 residual
pinned against the reference's own golden outputs and against the checks of
tests/cpu_fp64_residual/test_cpu_fp64_residual.cpp (restated here)."""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from tests.golden.make_golden import RES_CASES, gen_case, residual

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def test_residual_matches_reference_golden():
    with open(os.path.join(GOLD, "residual_ref.json")) as f:
        gold = json.load(f)
    assert len(gold) == len(RES_CASES)
    for g in gold:
        c = {k: g[k] for k in ("n", "lda", "kind", "dtype", "tile", "seed")}
        got = residual(c, "oracle")
        want = g["value"]
        if np.isinf(want):
            assert np.isinf(got), c
        else:
            assert got == pytest.approx(want, rel=1e-12, abs=1e-300), c


def test_residual_matches_reference_live():
    """Same cases against the reference header compiled in place (when present)."""
    if oracle.ref_lib() is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    for c in RES_CASES[::7]:
        a, b = residual(c, "oracle"), residual(c, "ref")
        assert (np.isinf(a) and np.isinf(b)) or a == pytest.approx(b, rel=1e-12), c


def _long_double_reference(factor, original, perm, n, lda, cholesky):
    """Unblocked oracle (test_cpu_fp64_residual.cpp:25-49) in extended precision."""
    num = np.longdouble(0)
    den = np.longdouble(0)
    F = np.asarray(factor, dtype=np.longdouble)
    for j in range(n):
        for i in range(n):
            prod = np.longdouble(0)
            for k in range(n):
                left = 0 if i < k else (1 if (not cholesky and i == k) else F[k * lda + i])
                if cholesky:
                    right = 0 if j < k else F[k * lda + j]
                else:
                    right = 0 if k > j else F[j * lda + k]
                prod += np.longdouble(left) * np.longdouble(right)
            a = np.longdouble(original[j * lda + perm[i]])
            num += (prod - a) ** 2
            den += a * a
    return float(np.sqrt(num / den))


@pytest.mark.parametrize("n", [1, 2, 3, 5, 11])
@pytest.mark.parametrize("padding", [0, 3])
@pytest.mark.parametrize("cholesky,pivoting", [(False, False), (False, True), (True, False)])
def test_layouts_tiles_permutation(n, padding, cholesky, pivoting):
    """test_cpu_fp64_residual.cpp:51-107: layouts, lda padding, 3-cycle pivots, tiles."""
    lda = n + padding
    factor = np.full(lda * n, np.nan, dtype=np.float32)
    original = np.zeros(lda * n, dtype=np.float32)
    pivots = np.arange(1, n + 1, dtype=np.int32)
    perm = list(range(n))
    if pivoting and n >= 3:
        pivots[0] = 3
        pivots[1] = 3
        for k in range(n):
            p = pivots[k] - 1
            perm[k], perm[p] = perm[p], perm[k]
    for j in range(n):
        for i in range(n):
            if not cholesky or i >= j:
                factor[j * lda + i] = np.float32(0.13) * np.float32(i + 1) - np.float32(0.07) * np.float32(j + 1) + (np.float32(2) if i == j else np.float32(0))
    for j in range(n):
        for i in range(n):
            prod = np.longdouble(0)
            for k in range(min(i, j) + 1):
                l = 1.0 if (not cholesky and i == k) else factor[k * lda + i]
                r = factor[k * lda + j] if cholesky else factor[j * lda + k]
                prod += np.longdouble(l) * np.longdouble(r)
            original[j * lda + perm[i]] = np.float32(prod)
    expected = _long_double_reference(factor, original, perm, n, lda, cholesky)
    for tile in (1, 2, 3, 4, 512):
        if cholesky:
            got = oracle.potrf_residual(factor, original, n, lda, tile)
        else:
            got = oracle.getrf_residual(factor, original, pivots, n, lda, pivoting, tile)
        tol = max(1e-18, abs(expected) * 1e-7)
        assert np.isfinite(got) and abs(got - expected) <= tol


def test_precision_and_errors():
    """test_cpu_fp64_residual.cpp:109-147."""
    f = np.nextafter(np.float32(1), np.float32(2))
    o = np.float32(f * f)
    exact = np.longdouble(f) * np.longdouble(f)
    r = oracle.potrf_residual(np.array([f]), np.array([o]), 1, 1)
    assert r > 0
    assert r == pytest.approx(float(abs(exact - np.longdouble(o)) / np.longdouble(o)), rel=1e-7)
    z, one = np.array([0], np.float32), np.array([1], np.float32)
    assert oracle.potrf_residual(z, z, 1, 1) == 0
    assert np.isinf(oracle.potrf_residual(one, z, 1, 1))
    assert np.isinf(oracle.potrf_residual(np.array([np.nan], np.float32), one, 1, 1))
    assert np.isinf(oracle.getrf_residual(one, one, np.array([0], np.int32), 1, 1, True))
    for tile in (0, -1):
        with pytest.raises(ValueError):
            oracle.potrf_residual(one, one, 1, 1, tile)
    big = oracle.getrf_residual(np.array([1e160]), np.array([2e160]), None, 1, 1, False)
    assert big == pytest.approx(0.5, rel=1e-7)
    small = oracle.getrf_residual(np.array([1e-200]), np.array([2e-200]), None, 1, 1, False)
    assert small == pytest.approx(0.5, rel=1e-7)


def test_seed_parser():
    """test_cpu_fp64_residual.cpp:149-165 (seed.h:5-19)."""
    assert oracle.parse_seed("0") == (True, 0)
    assert oracle.parse_seed("4294967295") == (True, 4294967295)
    for text in ("", "-1", "+1", "1x", "4294967296"):
        ok, v = oracle.parse_seed(text)
        assert not ok and v == 19
    assert not oracle.parse_seed(None)[0]


def test_reference_unit_test_binary_passes():
    """Run the reference's own 170-check test compiled in place (oracle/_ref)."""
    exe = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "test_cpu_fp64_residual")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref not built")
    p = subprocess.run([exe], capture_output=True, text=True)
    assert p.returncode == 0 and "PASS: 170 checks" in p.stdout


def test_blas_residual_agrees_with_c_oracle():
    for n in (7, 33, 96):
        A = oracle.spd_gram(n, 3)
        L, info = oracle.double_blocked_potrf(A, 32, 8)
        assert info == 0
        a = oracle.potrf_residual(L.ravel(order="F"), np.asfortranarray(A).ravel(order="F"), n, n)
        b = oracle.potrf_residual_blas(L, A)
        assert a == pytest.approx(b, rel=1e-9)
        G = oracle.general_uniform(n, 4)
        LU, ipiv, info = oracle.double_blocked_getrf(G, 32, 8)
        a = oracle.getrf_residual(LU.ravel(order="F"), G.ravel(order="F"), ipiv, n, n)
        b = oracle.getrf_residual_blas(LU, G, ipiv)
        assert a == pytest.approx(b, rel=1e-9)


@pytest.mark.parametrize("n,block", [(1, 4), (7, 3), (96, 32), (301, 64), (300, 512)])
def test_tiled_residuals_agree_with_c_oracle(n, block):
    """The block-column BLAS residuals used at n >= 8192 give the C oracle's
    value (both triangles of A compared, ragged last block, block > n)."""
    A = oracle.spd_gram(n, 3)
    L, info = oracle.double_blocked_potrf(A, 32, 8)
    assert info == 0
    L = np.asfortranarray(L)
    a = oracle.potrf_residual(L.ravel(order="F"), np.asfortranarray(A).ravel(order="F"), n, n)
    assert oracle.potrf_residual_tiled(L, A, block) == pytest.approx(a, rel=1e-9, abs=1e-300)
    # a non-symmetric "original": the upper triangle is compared with (L L^T)^T
    rng = np.random.default_rng(n)
    A2 = (A + np.triu(rng.standard_normal((n, n)), 1).astype(np.float32) * 1e-3).astype(np.float32)
    a2 = oracle.potrf_residual(L.ravel(order="F"), np.asfortranarray(A2).ravel(order="F"), n, n)
    assert oracle.potrf_residual_tiled(L, A2, block) == pytest.approx(a2, rel=1e-9)
    G = oracle.general_uniform(n, 4)
    LU, ipiv, info = oracle.double_blocked_getrf(G, 32, 8)
    a = oracle.getrf_residual(LU.ravel(order="F"), G.ravel(order="F"), ipiv, n, n)
    assert oracle.getrf_residual_tiled(LU, G, ipiv, block) == pytest.approx(a, rel=1e-9,
                                                                             abs=1e-300)


def test_tiled_residual_edge_cases():
    n = 40
    G = oracle.general_uniform(n, 4)
    LU, ipiv, _ = oracle.double_blocked_getrf(G, 16, 8)
    bad = ipiv.copy()
    bad[5] = 3  # ipiv[r] < r + 1: invalid
    assert np.isinf(oracle.getrf_residual_tiled(LU, G, bad, 16))
    LU2 = LU.copy()
    LU2[30, 31] = np.nan
    assert np.isinf(oracle.getrf_residual_tiled(LU2, G, ipiv, 16))
    Z = np.zeros((n, n), np.float32)
    assert oracle.potrf_residual_tiled(Z, Z, 16) == 0.0


@pytest.mark.parametrize("n,nb,b", [(200, 64, 16), (300, 128, 32), (97, 40, 7)])
def test_c_double_blocked_loops_match_lapack(n, nb, b):
    """The reference schedules restated in C reproduce host LAPACK's pivots and
    stay within the scaled-residual bound."""
    A = oracle.spd_gram(n, 0)
    L, info = oracle.double_blocked_potrf(A, nb, b, syrk_k_tile=nb // 2)
    assert info == 0 and oracle.scaled(oracle.potrf_residual_blas(L, A), n) <= 10
    G = oracle.general_uniform(n, 1)
    LU, ipiv, info = oracle.double_blocked_getrf(G, nb, b)
    _, ipiv_l, info_l = oracle.lapack_sgetrf(G)
    assert info == info_l == 0
    np.testing.assert_array_equal(ipiv, ipiv_l)
    assert oracle.scaled(oracle.getrf_residual_blas(LU, G, ipiv), n) <= 10


def test_lapack_golden_pivots_reproduce():
    """Committed host-sgetrf pivots (tests/golden/lapack_f32.npz) match a live run."""
    g = np.load(os.path.join(GOLD, "lapack_f32.npz"))
    for n in (64, 256, 512):
        _, ipiv, info = oracle.lapack_sgetrf(oracle.general_uniform(n, 1))
        np.testing.assert_array_equal(ipiv, g[f"getrf_ipiv_{n}"])
        assert g[f"getrf_scaled_{n}"] <= 10 and g[f"potrf_scaled_{n}"] <= 10


def test_generator_values():
    u = oracle.uniform_pm1(1 << 16, 7)
    assert u.dtype == np.float32 and u.min() >= -1 and u.max() < 1
    assert np.all((u.astype(np.float64) + 1) * 2 ** 23 == np.round((u.astype(np.float64) + 1) * 2 ** 23))
    assert abs(float(u.mean())) < 0.01
    np.testing.assert_array_equal(oracle.uniform_pm1(10, 7, offset=5), u[5:15])
    A = oracle.spd_gram(64, 0)
    np.testing.assert_array_equal(A, A.T)
    assert np.linalg.eigvalsh(A.astype(np.float64)).min() > 0.9


@pytest.mark.parametrize("n,nb,b", [(200, 64, 16), (300, 128, 32), (97, 40, 7), (1, 8, 4)])
def test_c_double_blocked_loops_f64_match_lapack(n, nb, b):
    """The FP64 twins of the restated loops reproduce host LAPACK dpotrf /
    dgetrf: factors to FP64 rounding, identical pivots, info on failure."""
    from scipy.linalg import lapack
    G = oracle.general_uniform(n, 0).astype(np.float64)
    A = G @ G.T / n + np.eye(n)
    A = 0.5 * (A + A.T)
    L, info = oracle.double_blocked_potrf_f64(A, nb, b, syrk_k_tile=nb // 2)
    ref, rinfo = lapack.dpotrf(np.asfortranarray(A), lower=1, clean=1)
    assert info == rinfo == 0
    assert np.abs(np.tril(L) - ref).max() <= 1e-13 * np.abs(ref).max()
    M = oracle.general_uniform(n, 1).astype(np.float64)
    LU, ipiv, info = oracle.double_blocked_getrf_f64(M, nb, b)
    lu_l, ipiv_l, info_l = oracle.lapack_dgetrf(M)
    assert info == info_l == 0
    np.testing.assert_array_equal(ipiv, ipiv_l)
    assert np.abs(LU - lu_l).max() <= 1e-12 * np.abs(lu_l).max()
    # a failing column: same info as LAPACK
    if n > 50:
        A[50, 50] = -1.0
        _, info = oracle.double_blocked_potrf_f64(A, nb, b)
        _, rinfo = lapack.dpotrf(np.asfortranarray(A), lower=1)
        assert info == rinfo == 51
        M[:, 30] = 0.0
        _, _, info = oracle.double_blocked_getrf_f64(M, nb, b)
        assert info == oracle.lapack_dgetrf(M)[2] == 31


@pytest.mark.parametrize("n,nb,b", [(200, 64, 16), (300, 128, 32), (97, 40, 7), (256, 256, 64),
                                    (1, 8, 4)])
def test_batched_pivot_schedule_equals_immediate(n, nb, b):
    """The batched-pivot schedule (interchanges deferred to the block's columns,
    then to earlier and next-block columns at the end of each outer block)
    moves the same data as applying every panel's swaps at once: factors and
    pivots are bit-identical to the immediate-pivot loop in FP32 and FP64,
    and the pivots are host LAPACK's."""
    G = oracle.general_uniform(n, 1)
    LU_i, ipiv_i, info_i = oracle.double_blocked_getrf(G, nb, b)
    LU_b, ipiv_b, info_b = oracle.double_blocked_getrf_batched(G, nb, b)
    np.testing.assert_array_equal(LU_b, LU_i)
    np.testing.assert_array_equal(ipiv_b, ipiv_i)
    assert info_b == info_i == 0
    np.testing.assert_array_equal(ipiv_b, oracle.lapack_sgetrf(G)[1])
    G64 = G.astype(np.float64)
    LU_i, ipiv_i, _ = oracle.double_blocked_getrf_f64(G64, nb, b)
    LU_b, ipiv_b, _ = oracle.double_blocked_getrf_batched(G64, nb, b, dtype=np.float64)
    np.testing.assert_array_equal(LU_b, LU_i)
    np.testing.assert_array_equal(ipiv_b, oracle.lapack_dgetrf(G64)[1])


@pytest.mark.parametrize("n,nb", [(200, 48), (97, 32), (1, 4), (130, 130)])
def test_right_looking_baselines_match_lapack(n, nb):
    """The right-looking POTRF / GETRF baselines and the NPVT variant restated
    in C: Cholesky factors and info as host LAPACK (FP32 within the scaled
    residual bound, FP64 to rounding), LU pivots identical to sgetrf/dgetrf,
    NPVT equal to LAPACK's LU when diagonal dominance makes the pivots the
    identity."""
    from scipy.linalg import lapack
    A = oracle.spd_gram(n, 0)
    L, info = oracle.blocked_right_looking_potrf(A, nb)
    assert info == 0 and oracle.scaled(oracle.potrf_residual_blas(L, A), n) <= 10
    A64 = A.astype(np.float64)
    L64, info = oracle.blocked_right_looking_potrf(A64, nb, dtype=np.float64)
    ref, rinfo = lapack.dpotrf(np.asfortranarray(A64), lower=1, clean=1)
    assert info == rinfo == 0
    assert np.abs(np.tril(L64) - ref).max() <= 1e-13 * np.abs(ref).max()
    G = oracle.general_uniform(n, 1)
    LU, ipiv, info = oracle.blocked_right_looking_getrf(G, nb)
    assert info == 0
    np.testing.assert_array_equal(ipiv, oracle.lapack_sgetrf(G)[1])
    assert oracle.scaled(oracle.getrf_residual_blas(LU, G, ipiv), n) <= 10
    G64 = G.astype(np.float64)
    LU64, ipiv64, _ = oracle.blocked_right_looking_getrf(G64, nb, dtype=np.float64)
    lu_l, ipiv_l, _ = oracle.lapack_dgetrf(G64)
    np.testing.assert_array_equal(ipiv64, ipiv_l)
    assert np.abs(LU64 - lu_l).max() <= 1e-12 * np.abs(lu_l).max()
    D = G64 + n * np.eye(n)
    LUn, _, info = oracle.blocked_right_looking_getrf(D, nb, pivot=False, dtype=np.float64)
    lu_d, piv_d, _ = oracle.lapack_dgetrf(D)
    assert info == 0 and np.array_equal(piv_d, np.arange(1, n + 1))
    assert np.abs(LUn - lu_d).max() <= 1e-13 * np.abs(lu_d).max()


@pytest.mark.parametrize("n,nb", [(200, 48), (97, 32), (1, 4), (300, 64)])
def test_recursive_potrf_matches_lapack(n, nb):
    """The recursive Cholesky restated in C: factors as host LAPACK (FP32
    within the scaled residual bound, FP64 to rounding) and LAPACK's info for
    a matrix with a failing column."""
    from scipy.linalg import lapack
    A = oracle.spd_gram(n, 5)
    L, info = oracle.recursive_potrf(A, nb)
    assert info == 0 and oracle.scaled(oracle.potrf_residual_blas(L, A), n) <= 10
    A64 = A.astype(np.float64)
    L64, info = oracle.recursive_potrf(A64, nb, dtype=np.float64)
    ref, rinfo = lapack.dpotrf(np.asfortranarray(A64), lower=1, clean=1)
    assert info == rinfo == 0
    assert np.abs(np.tril(L64) - ref).max() <= 1e-13 * np.abs(ref).max()
    if n > 80:
        A64[80, 80] = -1.0
        _, info = oracle.recursive_potrf(A64, nb, dtype=np.float64)
        assert info == lapack.dpotrf(np.asfortranarray(A64), lower=1)[1] == 81


def test_pivot_agreement_rules():
    """pivot_agreement: identical sequences; an exact tie (either row is a
    correct partial-pivoting choice); a clear gap; and the rounding-scale rule
    against the relative gap pivot_divergence reports."""
    A = np.array([[1.0, 2.0, 0.5], [-1.0, 3.0, 1.0], [0.25, 1.0, 4.0]], dtype=np.float32)
    assert oracle.pivot_agreement(A, [1, 2, 3], [1, 2, 3]) == {"first_divergence": None,
                                                              "near_tie": True}
    tie = oracle.pivot_agreement(A, [1, 2, 3], [2, 2, 3])  # |1| == |-1| in column 0
    assert tie["first_divergence"] == 0 and tie["rel_gap"] == 0.0 and tie["near_tie"]
    B = np.array([[1.0, 2.0], [4.0, 1.0]], dtype=np.float32)
    far = oracle.pivot_agreement(B, [2, 2], [1, 2])
    assert far["first_divergence"] == 0 and not far["near_tie"]
    assert abs(far["rel_gap"] - 0.75) < 1e-12
    # column 1 after a common first pivot: same gap as pivot_divergence
    rng = np.random.default_rng(4)
    C = rng.uniform(-1, 1, (6, 6)).astype(np.float32)
    _, ref, _ = oracle.lapack_sgetrf(C)
    other = ref.copy()
    other[1] = 6 if ref[1] != 6 else 5
    pa = oracle.pivot_agreement(C, ref, other)
    j, gap = oracle.pivot_divergence(C, ref, other)
    assert pa["first_divergence"] == j == 1 and abs(pa["rel_gap"] - gap) < 1e-12
    assert pa["gap_over_rounding"] > 0
