"""CPU tests of the selector's host logic and of its FP64 oracle (the numpy
restatement of the network, its gradient and Adam)."""
import numpy as np

import oracle
from oracle import mlp
from hygondoubleblockedfactorizations_b200 import selector as sel


def rand_problem(N=37, seed=0):
    rng = np.random.default_rng(seed)
    F, K = sel.FEATURES, sel.NUM_CLASSES
    X = rng.uniform(-1, 1, size=(N, F)).astype(np.float32)
    kinds = rng.integers(0, 3, size=N)
    mask = np.zeros((N, K), np.float32)
    for i, kd in enumerate(kinds):
        kind = ("blocks", "panel", "variant")[kd]
        mask[i] = [1.0 if c[0] == kind else 0.0 for c in sel.CANDIDATES]
    T = np.where(mask > 0, rng.uniform(1.0, 1.3, size=(N, K)), np.inf)
    Q = sel.soft_targets(T, mask)
    return X, T, Q, mask


def test_oracle_gradient_matches_finite_differences():
    F, K = sel.FEATURES, sel.NUM_CLASSES
    X, T, Q, mask = rand_problem()
    theta = mlp.init_params(F, K, seed=5).astype(np.float64)
    theta[F * 64:F * 64 + 64] = 0.05  # non-zero biases so every ReLU path is exercised
    loss, g = mlp.loss_and_grad(theta, X, Q, mask, F, K)
    assert np.isfinite(loss) and loss > 0
    rng = np.random.default_rng(1)
    idx = rng.choice(len(theta), size=40, replace=False)
    num = mlp.numeric_grad(theta, X, Q, mask, F, K, idx)
    assert np.allclose(num, g[idx], rtol=1e-5, atol=1e-8)


def test_soft_targets_and_regret():
    X, T, Q, mask = rand_problem(20, 2)
    assert np.allclose(Q.sum(1), 1.0, atol=1e-6)
    assert np.all(Q[mask == 0] == 0)
    assert np.allclose(Q, mlp.soft_targets(T, mask), atol=1e-6)
    best = np.argmin(np.where(mask > 0, T, np.inf), axis=1)
    assert np.all(np.argmax(Q, axis=1) == best)
    assert np.allclose(sel.regret(best, T), 0.0)
    d = sel.default_classes(mask)
    assert np.all(mask[np.arange(len(d)), d] > 0)


def test_features_and_masks():
    f = sel.features("potrf", "fp32", [4096])
    assert f.shape == (sel.FEATURES,) and f[0] == f[1] == 12 / 16 and f[2] == 0 and f[4] == 0
    assert f[6] == 1 and f[9] == 1 and f[5] == 0
    g = sel.features("batched", "fp32", [16, 512], 0.5)
    assert g[11] == 1 and g[5] == 0.5 and g[2] == 1 / 16
    assert sel.valid_mask("getrf", "fp32")[:5].sum() == 5
    assert sel.valid_mask("potrf", "bf16")[5:8].sum() == 3
    assert sel.valid_mask("batched", "fp32")[8:].sum() == 3


def test_dataset_and_split():
    recs = [{"op": "potrf", "precision": "fp32", "ns": [1024], "times": {"0": 2.0, "3": 1.0}},
            {"op": "getrf", "precision": "bf16", "ns": [1536], "times": {"5": 1.0, "6": 1.5}},
            {"op": "batched", "precision": "fp32", "ns": [20, 40], "lu_fraction": 0.5,
             "heldout": True, "times": {"8": 3.0, "9": 2.0, "10": 2.5}}]
    X, T, M = sel.dataset(recs)
    assert X.shape == (3, sel.FEATURES) and M[0].sum() == 2 and np.isinf(T[0, 1])
    train, test = sel.split_heldout(recs)
    assert len(train) == 1 and len(test) == 2


def test_oracle_init_uses_counter_stream():
    F, K = sel.FEATURES, sel.NUM_CLASSES
    th = mlp.init_params(F, K, seed=3)
    u = oracle.uniform_pm1(mlp.n_params(F, K), 3)
    s1 = np.sqrt(np.float32(6.0) / np.float32(F + 64)).astype(np.float32)
    assert th[0] == np.float32(u[0] * s1)
    assert th[F * 64] == 0.0 and len(th) == mlp.n_params(F, K)


def test_measured_records_fixture():
    import json
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "selector_records_b200.json")
    recs = json.load(open(path))
    train, test = sel.split_heldout(recs)
    X, T, M = sel.dataset(train)
    Xt, Tt, Mt = sel.dataset(test)
    assert len(train) == 240 and len(test) == 202
    assert np.all(np.isfinite(X)) and np.all(M.sum(1) >= 3)
    # every measured row has a finite optimum among its valid candidates
    assert np.all(np.isfinite(np.where(M > 0, T, np.inf).min(1)))
