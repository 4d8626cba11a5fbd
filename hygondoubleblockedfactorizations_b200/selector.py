"""Learned configuration selector: a 3-layer FP32 MLP (64 hidden units) that
maps a problem description to one of the candidate configurations the
exhaustive autotuner (``tuner``) measures, with a confidence score.

Problem features (F = 12, ``features``): log2 of the mean and of the largest
order, log2 of the matrix count, the mean order / 16384, the coefficient of
variation of the orders, the LU fraction, one-hot precision (fp32, bf16,
fp16) and one-hot operation (potrf, getrf, batched).

Candidates (K = 11, ``CANDIDATES``): the FP32 double-blocked (outer, inner)
block pairs of ``tuner.POTRF_GRID``, the mixed-precision panel widths and the
CTA-size variants of the persistent batched kernel.  A per-sample mask marks
the candidates that apply (blocks for FP32 POTRF/GETRF, panel widths for
BF16/FP16, variants for batched work).

Training targets are soft: q_k ~ exp(-(t_k / t_best - 1) / tau) over the valid
candidates, so the fastest candidate dominates and near-ties share the mass.
Forward, backward and the Adam steps run in this library's own CUDA kernels
(``hdbf_selector_*``); nothing here computes on the host but the features.

``choose`` returns the selected candidate, its confidence, and whether the
confidence fell below the threshold, in which case the caller should use the
fallback (``DEFAULTS``, or an exhaustive ``tuner`` run).
"""
from __future__ import annotations

import ctypes
import json
import math

import numpy as np

from . import lib, status_string, HdbfError

HIDDEN = 64
FEATURES = 12
OPS = ("potrf", "getrf", "batched")
PRECISIONS = ("fp32", "bf16", "fp16")

# (kind, parameters): blocks = (outer, inner); panel = (width,); variant = (index,)
CANDIDATES = [
    ("blocks", (2048, 256)), ("blocks", (4096, 256)), ("blocks", (4096, 512)),
    ("blocks", (8192, 512)), ("blocks", (8192, 1024)),
    ("panel", (256,)), ("panel", (512,)), ("panel", (1024,)),
    ("variant", (0,)), ("variant", (1,)), ("variant", (2,)),
]
NUM_CLASSES = len(CANDIDATES)
# Fixed policies used when the selector is not confident.
DEFAULTS = {"blocks": 3, "panel": 6, "variant": 9}


def candidate_kind(op: str, precision: str) -> str:
    if op == "batched":
        return "variant"
    return "blocks" if precision == "fp32" else "panel"


def valid_mask(op: str, precision: str) -> np.ndarray:
    kind = candidate_kind(op, precision)
    return np.array([1.0 if c[0] == kind else 0.0 for c in CANDIDATES], dtype=np.float32)


def order_stats(ns) -> dict:
    """The size-histogram moments the features use."""
    ns = np.atleast_1d(np.asarray(ns, dtype=np.float64))
    return {"count": int(len(ns)), "mean": float(ns.mean()), "max": float(ns.max()),
            "std": float(ns.std())}


def features(op: str, precision: str, ns=None, lu_fraction: float | None = None,
             stats: dict | None = None) -> np.ndarray:
    st = stats if stats is not None else order_stats(ns)
    mean, top, cnt = st["mean"], st["max"], st["count"]
    if lu_fraction is None:
        lu_fraction = 1.0 if op == "getrf" else 0.0
    f = np.zeros(FEATURES, dtype=np.float32)
    f[0] = math.log2(mean) / 16.0
    f[1] = math.log2(top) / 16.0
    f[2] = math.log2(cnt) / 16.0
    f[3] = mean / 16384.0
    f[4] = st["std"] / mean
    f[5] = lu_fraction
    f[6 + PRECISIONS.index(precision)] = 1.0
    f[9 + OPS.index(op)] = 1.0
    return f


def soft_targets(times: np.ndarray, mask: np.ndarray, tau: float = 0.02) -> np.ndarray:
    t = np.where(mask > 0, times, np.inf)
    best = t.min(axis=1, keepdims=True)
    s = np.where(np.isfinite(t), np.exp(-(t / best - 1.0) / tau), 0.0)
    return (s / s.sum(axis=1, keepdims=True)).astype(np.float32)


def dataset(records):
    """records: dicts {op, precision, ns or stats, lu_fraction?, times: {class: ms}}
    -> (X [N,F], T [N,K] with inf where not measured, mask [N,K])."""
    X, T, M = [], [], []
    for r in records:
        X.append(features(r["op"], r["precision"], r.get("ns"), r.get("lu_fraction"),
                          r.get("stats")))
        m = valid_mask(r["op"], r["precision"])
        t = np.full(NUM_CLASSES, np.inf)
        for k, ms in r["times"].items():
            t[int(k)] = float(ms)
        m = np.where(np.isfinite(t), m, 0.0).astype(np.float32)
        T.append(t)
        M.append(m)
    return np.array(X, np.float32), np.array(T), np.array(M, np.float32)


def regret(cls: np.ndarray, T: np.ndarray) -> np.ndarray:
    best = np.where(np.isfinite(T), T, np.inf).min(axis=1)
    return T[np.arange(len(cls)), cls] / best - 1.0


def default_classes(mask: np.ndarray) -> np.ndarray:
    out = []
    for m in mask:
        kinds = {CANDIDATES[k][0] for k in np.nonzero(m > 0)[0]}
        kind = kinds.pop() if len(kinds) == 1 else "blocks"
        d = DEFAULTS[kind]
        out.append(d if m[d] > 0 else int(np.argmax(m)))
    return np.array(out)


class Selector:
    """Device-resident selector parameters plus Adam state."""

    def __init__(self, torch, handle, seed: int = 0):
        self.torch = torch
        self.handle = handle
        self.P = lib().hdbf_selector_num_params(FEATURES, NUM_CLASSES)
        dev = "cuda"
        self.theta = torch.zeros(self.P, dtype=torch.float32, device=dev)
        self.m = torch.zeros_like(self.theta)
        self.v = torch.zeros_like(self.theta)
        self.steps = 0
        self._check(lib().hdbf_selector_init(handle.ptr, self._p(self.theta), FEATURES,
                                             NUM_CLASSES, seed), "selector_init")

    @staticmethod
    def _p(t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else None

    @staticmethod
    def _check(st, what):
        if st != 0:
            raise HdbfError(f"{what}: {status_string(st)}")

    def _dev(self, a):
        return self.torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()

    def loss_grad(self, X, Q, mask):
        """Loss and gradient at the current parameters (no update)."""
        torch = self.torch
        dX, dQ, dM = self._dev(X), self._dev(Q), self._dev(mask)
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        grad = torch.zeros(self.P, dtype=torch.float32, device="cuda")
        self._check(lib().hdbf_selector_train(
            self.handle.ptr, self._p(self.theta), None, None, 0, self._p(dX), self._p(dQ),
            self._p(dM), len(X), FEATURES, NUM_CLASSES, 0, 0.0, 0.0, self._p(loss),
            self._p(grad)), "selector_train")
        torch.cuda.synchronize()
        return float(loss.item()), grad.cpu().numpy()

    def fit(self, X, T, mask, epochs=3000, lr=3e-3, weight_decay=1e-4, tau=0.02):
        """Full-batch Adam on soft targets from times T; returns the losses."""
        torch = self.torch
        Q = soft_targets(T, mask, tau)
        dX, dQ, dM = self._dev(X), self._dev(Q), self._dev(mask)
        losses = torch.zeros(epochs, dtype=torch.float32, device="cuda")
        self._check(lib().hdbf_selector_train(
            self.handle.ptr, self._p(self.theta), self._p(self.m), self._p(self.v), self.steps,
            self._p(dX), self._p(dQ), self._p(dM), len(X), FEATURES, NUM_CLASSES, epochs,
            float(lr), float(weight_decay), self._p(losses), None), "selector_train")
        self.steps += epochs
        torch.cuda.synchronize()
        return losses.cpu().numpy()

    def predict(self, X, mask):
        torch = self.torch
        N = len(X)
        dX, dM = self._dev(X), self._dev(mask)
        cls = torch.zeros(N, dtype=torch.int32, device="cuda")
        conf = torch.zeros(N, dtype=torch.float32, device="cuda")
        probs = torch.zeros(N * NUM_CLASSES, dtype=torch.float32, device="cuda")
        self._check(lib().hdbf_selector_predict(
            self.handle.ptr, self._p(self.theta), self._p(dX), self._p(dM), N, FEATURES,
            NUM_CLASSES, self._p(cls), self._p(conf), self._p(probs)), "selector_predict")
        torch.cuda.synchronize()
        return cls.cpu().numpy(), conf.cpu().numpy(), probs.cpu().numpy().reshape(N, NUM_CLASSES)

    def choose(self, op, precision, ns, threshold=0.4, lu_fraction=None):
        """(candidate, confidence, fell_back): the fixed default when the
        confidence is below the threshold."""
        X = features(op, precision, ns, lu_fraction)[None]
        m = valid_mask(op, precision)[None]
        cls, conf, _ = self.predict(X, m)
        k, c = int(cls[0]), float(conf[0])
        if c < threshold:
            return CANDIDATES[int(default_classes(m)[0])], c, True
        return CANDIDATES[k], c, False

    def state(self) -> dict:
        return {"features": FEATURES, "classes": NUM_CLASSES, "hidden": HIDDEN,
                "theta": self.theta.cpu().numpy().tolist()}

    def load(self, state: dict):
        assert state["features"] == FEATURES and state["classes"] == NUM_CLASSES
        self.theta.copy_(self.torch.tensor(state["theta"], dtype=self.torch.float32))


def evaluate(sel: Selector, X, T, mask, threshold=0.4):
    """Regret of the selector alone, with fallback to the exhaustive tuner
    below the threshold (regret 0, tuning cost paid), and of the defaults."""
    cls, conf, _ = sel.predict(X, mask)
    r_mlp = regret(cls, T)
    low = conf < threshold
    r_fb = np.where(low, 0.0, r_mlp)
    r_def = regret(default_classes(mask), T)
    return {"samples": int(len(X)), "mean_regret": float(r_mlp.mean()),
            "max_regret": float(r_mlp.max()), "p90_regret": float(np.quantile(r_mlp, 0.9)),
            "mean_regret_with_fallback": float(r_fb.mean()), "fallback_rate": float(low.mean()),
            "default_mean_regret": float(r_def.mean()), "default_max_regret": float(r_def.max()),
            "exact_best_rate": float((r_mlp <= 1e-12).mean())}


def split_heldout(records):
    """Held out: single-matrix orders n = 512 (mod 1024) and batched mixes
    flagged ``heldout``; the rest train."""
    train, test = [], []
    for r in records:
        if r["op"] == "batched":
            (test if r.get("heldout") else train).append(r)
        else:
            n = int(r["stats"]["max"]) if "stats" in r else int(np.atleast_1d(r["ns"])[0])
            (test if n % 1024 == 512 else train).append(r)
    return train, test


def _main():
    import argparse
    import torch
    from . import Handle
    from . import tuner

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect", help="time every candidate on the tuning grid")
    c.add_argument("--out", required=True)
    c.add_argument("--nmax", type=int, default=32768)
    c.add_argument("--step", type=int, default=1024)
    c.add_argument("--mixes", type=int, default=48)
    c.add_argument("--heldout-mixes", type=int, default=16)
    e = sub.add_parser("evaluate", help="train on the grid, report held-out regret")
    e.add_argument("--records", required=True)
    e.add_argument("--epochs", type=int, default=3000)
    e.add_argument("--threshold", type=float, default=0.4)
    e.add_argument("--out")
    a = ap.parse_args()
    h = Handle(torch.cuda.current_stream().cuda_stream)
    if a.cmd == "collect":
        recs = tuner.collect(torch, h, a.nmax, a.step, a.mixes, a.heldout_mixes, log=print)
        with open(a.out, "w") as f:
            json.dump(recs, f)
    else:
        recs = json.load(open(a.records))
        train, test = split_heldout(recs)
        Xtr, Ttr, Mtr = dataset(train)
        Xte, Tte, Mte = dataset(test)
        sel = Selector(torch, h, seed=0)
        losses = sel.fit(Xtr, Ttr, Mtr, epochs=a.epochs)
        rep = {"train": evaluate(sel, Xtr, Ttr, Mtr, a.threshold),
               "heldout": evaluate(sel, Xte, Tte, Mte, a.threshold),
               "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
               "threshold": a.threshold, "epochs": a.epochs}
        for kind in ("blocks", "panel", "variant"):
            sel_rows = [i for i, m in enumerate(Mte) if m[[k for k, cnd in enumerate(CANDIDATES)
                                                           if cnd[0] == kind]].sum() > 0]
            if sel_rows:
                rep["heldout_" + kind] = evaluate(sel, Xte[sel_rows], Tte[sel_rows],
                                                  Mte[sel_rows], a.threshold)
        print(json.dumps(rep, indent=1))
        if a.out:
            with open(a.out, "w") as f:
                json.dump({"report": rep, "state": sel.state()}, f)


if __name__ == "__main__":
    _main()
