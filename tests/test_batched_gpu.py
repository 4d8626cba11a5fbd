"""GPU tests of the persistent batched factor-and-solve kernel (one launch for
the whole uneven batch) and of its autotuner.  Oracle: host LAPACK pivots
(with the near-tie rule), the C restatement of the reference's FP64 residual
(scaled by n * eps32, bound 10) and the FP64 backward error of each solution."""
import numpy as np
import pytest

import oracle
from hygondoubleblockedfactorizations_b200 import batch as bm
from hygondoubleblockedfactorizations_b200 import tuner

pytestmark = pytest.mark.gpu


def make_batch(torch, handle, n_spd=160, n_gen=80, seed=7):
    ops, ns = bm.config3_sizes(n_spd, n_gen, seed)
    b = bm.DeviceBatch(torch, ops, ns)
    bm.fill_batch(torch, handle, b, seed)
    return b


def check_batch(b, sample=None):
    worst = 0.0
    idx = range(b.count) if sample is None else sample
    info = b.info.cpu().numpy()
    for i in idx:
        n = int(b.ns[i])
        o = int(b.offsets[i])
        A0 = b.A0[o:o + n * n].cpu().numpy().reshape(n, n).T
        F = b.A[o:o + n * n].cpu().numpy().reshape(n, n).T
        r0 = int(b.roffsets[i])
        rhs = b.b0[r0:r0 + n].cpu().numpy().astype(np.float64)
        x = b.b[r0:r0 + n].cpu().numpy().astype(np.float64)
        assert info[i] == 0, (i, n, info[i])
        if b.ops[i] == 0:
            s = oracle.scaled(oracle.potrf_residual_blas(np.tril(F), A0), n)
        else:
            piv = b.ipiv_buf[r0:r0 + n].cpu().numpy()
            s = oracle.scaled(oracle.getrf_residual_blas(F, A0, piv), n)
            _, lp, _ = oracle.lapack_sgetrf(A0)
            pv = oracle.pivot_agreement(A0, lp, piv)
            assert pv["near_tie"], (i, n, pv)
        worst = max(worst, s)
        assert s <= 10.0, (i, n, s)
        be = oracle.backward_error(A0.astype(np.float64), x[:, None], rhs[:, None])
        assert be <= 50 * n * 2.0 ** -23, (i, n, be)
    return worst


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5])
def test_batched_variants(hd, handle, torch_cuda, variant):
    b = make_batch(torch_cuda, handle)
    st = b.run(handle, variant)
    torch_cuda.cuda.synchronize()
    assert st == 0 and handle.device_errors() == 0
    sample = list(range(0, b.count, 3))
    check_batch(b, sample)


def test_batched_replay_and_tuner(hd, handle, torch_cuda):
    b = make_batch(torch_cuda, handle, 64, 32, seed=9)
    best, times = tuner.tune_batched(torch_cuda, handle, b, reps=1)
    assert best in times and len(times) == hd.lib().hdbf_batched_num_variants() == 6
    bm.restore(b)
    st = b.run(handle, best)  # graph replay of the tuned variant
    torch_cuda.cuda.synchronize()
    assert st == 0
    check_batch(b)


def test_batched_not_positive_definite(hd, handle, torch_cuda):
    b = bm.DeviceBatch(torch_cuda, [0, 0], [40, 70])
    bm.fill_batch(torch_cuda, handle, b, 5)
    # make the second matrix indefinite at column 33
    M = b.matrix(1)
    M[33, 33] = -100.0
    b.A0 = b.A.clone()
    st = b.run(handle, 1)
    torch_cuda.cuda.synchronize()
    assert st == 0
    info = b.info.cpu().numpy()
    assert info[0] == 0 and info[1] == 34
