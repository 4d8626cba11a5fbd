"""GPU tests of the selector kernels (init, loss/gradient, Adam training,
prediction) against the FP64 numpy oracle, and of the selector's held-out
regret on a seeded synthetic timing model whose best configuration changes
with the order (and with the batch mix).

Tolerances: gradients and losses agree with the FP64 oracle to 1e-4 relative
(FP32 accumulation over <= a few hundred terms); after 60 Adam steps the
parameters agree to 2e-3 relative (Adam normalises each step, so FP32
rounding in the gradient moves a parameter by at most lr per step)."""
import numpy as np
import pytest

from oracle import mlp
from hygondoubleblockedfactorizations_b200 import selector as sel
from tests.test_selector_oracle import rand_problem

pytestmark = pytest.mark.gpu
F, K = sel.FEATURES, sel.NUM_CLASSES


def test_init_bit_identical(hd, handle, torch_cuda):
    s = sel.Selector(torch_cuda, handle, seed=11)
    assert np.array_equal(s.theta.cpu().numpy(), mlp.init_params(F, K, 11))


@pytest.mark.parametrize("N", [1, 31, 77])
def test_loss_and_gradient_match_oracle(hd, handle, torch_cuda, N):
    X, T, Q, mask = rand_problem(N, seed=N)
    s = sel.Selector(torch_cuda, handle, seed=2)
    th = s.theta.cpu().numpy()
    th[F * 64:F * 64 + 64] = 0.05
    s.theta.copy_(torch_cuda.tensor(th))
    loss, g = s.loss_grad(X, Q, mask)
    lo, go = mlp.loss_and_grad(th, X, Q, mask, F, K)
    assert abs(loss - lo) <= 1e-4 * abs(lo)
    assert np.abs(g - go).max() <= 1e-4 * np.abs(go).max()


def test_adam_training_matches_oracle(hd, handle, torch_cuda):
    X, T, Q, mask = rand_problem(70, seed=4)
    s = sel.Selector(torch_cuda, handle, seed=3)
    th0 = s.theta.cpu().numpy().astype(np.float64)
    losses = s.fit(X, T, mask, epochs=60, lr=1e-3, weight_decay=1e-4)
    th_o, losses_o = mlp.adam_train(th0, X, Q, mask, F, K, 60, 1e-3, 1e-4)
    assert np.allclose(losses, losses_o, rtol=2e-4)
    th = s.theta.cpu().numpy()
    assert np.abs(th - th_o).max() <= 2e-3 * np.abs(th_o).max()
    assert losses[-1] < losses[0]


def test_predict_matches_oracle_forward(hd, handle, torch_cuda):
    X, T, Q, mask = rand_problem(50, seed=6)
    s = sel.Selector(torch_cuda, handle, seed=8)
    s.fit(X, T, mask, epochs=200)
    cls, conf, probs = s.predict(X, mask)
    p, _ = mlp.forward(s.theta.cpu().numpy(), X, mask, F, K)
    assert np.allclose(probs, p, atol=1e-5)
    assert np.all(mask[np.arange(50), cls] > 0)
    assert np.allclose(conf, p.max(axis=1), atol=1e-5)


def synthetic_times(op, prec, ns, lu_frac, rng):
    """Cost model with crossovers inside the grid: larger blocks / wider
    panels / bigger CTAs cost less per flop but more per block."""
    ns = np.atleast_1d(np.asarray(ns, dtype=np.float64))
    kind = sel.candidate_kind(op, prec)
    t = {}
    if kind == "blocks":
        n = ns[0]
        a = [1.10, 1.06, 1.03, 1.0, 0.98]
        c = [0, 200, 400, 800, 1600]
        w = 2.0 if op == "getrf" else 1.0
        for k in range(5):
            t[k] = w * (a[k] * n ** 3 + c[k] * n ** 2) * 1e-9
    elif kind == "panel":
        n = ns[0]
        a = [1.06, 1.0, 0.97] if prec == "bf16" else [1.08, 1.0, 0.96]
        c = [0, 300, 900] if op == "potrf" else [0, 150, 600]
        for j, k in enumerate(range(5, 8)):
            t[k] = (a[j] * n ** 3 + c[j] * n ** 2) * 1e-9
    else:
        m = ns.mean()
        cost = (ns ** 3).sum()
        for j, k in enumerate(range(8, 11)):
            eff = [1.0 / (1 + (m / 150.0) ** 2), 1.0 / (1 + (m / 400.0) ** 2 + 0.15),
                   0.8 / (1 + 0.05 * (200.0 / m) ** 2)][j] * (1 + 0.3 * lu_frac * (j == 2))
            t[k] = cost / eff * 1e-9
    return {k: v * (1 + 0.005 * rng.standard_normal()) for k, v in t.items()}


def synthetic_records(seed=0):
    rng = np.random.default_rng(seed)
    recs = []
    for n in list(range(1024, 32769, 1024)) + list(range(1536, 32768, 1024)):
        for op in ("potrf", "getrf"):
            for prec in ("fp32", "bf16", "fp16"):
                recs.append({"op": op, "precision": prec, "ns": [n],
                             "times": synthetic_times(op, prec, [n], None, rng)})
    from hygondoubleblockedfactorizations_b200.tuner import random_mix
    for i in range(64):
        held = i >= 48
        ops, ns = random_mix(rng, held)
        recs.append({"op": "batched", "precision": "fp32", "ns": ns.tolist(), "heldout": held,
                     "lu_fraction": float(ops.mean()),
                     "times": synthetic_times("batched", "fp32", ns, float(ops.mean()), rng)})
    return recs


def test_selector_regret_on_heldout_orders_and_mixes(hd, handle, torch_cuda):
    train, test = sel.split_heldout(synthetic_records())
    Xtr, Ttr, Mtr = sel.dataset(train)
    Xte, Tte, Mte = sel.dataset(test)
    s = sel.Selector(torch_cuda, handle, seed=0)
    losses = s.fit(Xtr, Ttr, Mtr, epochs=3000)
    Q = sel.soft_targets(Ttr, Mtr)
    entropy = -np.where(Q > 0, Q * np.log(np.where(Q > 0, Q, 1.0)), 0.0).sum(1).mean()
    assert losses[-1] - entropy <= 0.2 * (losses[0] - entropy)  # near the loss floor
    rep = sel.evaluate(s, Xte, Tte, Mte)
    assert rep["mean_regret"] <= 0.05, rep
    assert rep["mean_regret"] < rep["default_mean_regret"], rep
    assert rep["mean_regret_with_fallback"] <= rep["mean_regret"] + 1e-12
    cand, conf, fell = s.choose("getrf", "fp32", [24576 + 512])
    assert cand[0] == "blocks" and 0 < conf <= 1 and fell == (conf < 0.4)


RECORDS = __import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                     "selector_records_b200.json")


def test_selector_regret_on_measured_b200_timings(hd, handle, torch_cuda):
    """Timings measured on a B200 by ``python -m hygondoubleblockedfactorizations_b200.selector
    collect`` (every candidate at n = 1024..32768 and n + 512, 64 batch mixes):
    the selector trained on the grid must stay within 5% of the exhaustive
    optimum on the held-out orders and mixes, and beat the fixed defaults."""
    import json
    train, test = sel.split_heldout(json.load(open(RECORDS)))
    Xtr, Ttr, Mtr = sel.dataset(train)
    Xte, Tte, Mte = sel.dataset(test)
    s = sel.Selector(torch_cuda, handle, seed=0)
    s.fit(Xtr, Ttr, Mtr, epochs=3000)
    rep = sel.evaluate(s, Xte, Tte, Mte)
    assert rep["mean_regret"] <= 0.05, rep
    assert rep["mean_regret"] < 0.5 * rep["default_mean_regret"], rep
    assert rep["mean_regret_with_fallback"] <= rep["mean_regret"] + 1e-12
