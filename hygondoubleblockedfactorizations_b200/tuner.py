"""Exhaustive autotuner.

* ``tune_batched`` times every launch shape of the persistent batched kernel
  (threads per CTA x panel width, ``hdbf_batched_variant_shape``) on a batch
  (inputs restored before each timed run) and returns the fastest.
* ``tune_blocks`` times a grid of (outer block, inner block) choices for the
  large double-blocked factorizations at one order n and returns the fastest.
* ``collect`` sweeps every candidate of the learned selector
  (``hygondoubleblockedfactorizations_b200.selector``) over the tuning grid:
  FP32 block pairs and BF16/FP16 panel widths for POTRF and GETRF at
  n = step, 2 step, ... and at the held-out orders n + step/2, plus the
  batched-kernel variants on random uneven mixes; its records are the
  selector's training and evaluation data.
Timings are CUDA-event device times after a warm-up run (the warm-up also
records the CUDA graph the library replays).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import batch as batch_mod
from . import PREC, call, lib


def _time(torch, fn, reps=2):
    fn()
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1)
        best = t if best is None else min(best, t)
    return best


def tune_batched(torch, handle, batch, reps=2):
    """Returns (best_variant, {variant: ms}) for the batched kernel."""
    res = {}
    for v in range(lib().hdbf_batched_num_variants()):
        def run(v=v):
            batch_mod.restore(batch)
            batch.run(handle, v)
        res[v] = _time(torch, run, reps)
    best = min(res, key=res.get)
    return best, res


# Candidate (outer, inner) blocks per operation; outer is clamped to n.
POTRF_GRID = [(2048, 256), (4096, 256), (4096, 512), (8192, 512), (8192, 1024)]
GETRF_GRID = [(2048, 256), (4096, 256), (4096, 512), (8192, 512), (8192, 1024)]


def tune_blocks(torch, handle, op, n, grid=None, reps=1):
    """Time the double-blocked factorization of order n for each (outer, inner)
    in the grid; returns a list of records {op, n, outer, inner, ms}."""
    grid = grid or (POTRF_GRID if op == "potrf" else GETRF_GRID)
    P = ctypes.c_void_p
    A0 = torch.empty(n * n, dtype=torch.float32, device="cuda")
    lib().hdbf_fill_uniform(handle.ptr, P(A0.data_ptr()), n * n, 11, 0)
    if op == "potrf":
        M = A0.view(n, n).double()
        S = M @ M.t() / n
        S.diagonal().add_(1.0)
        A0.copy_(S.float().reshape(-1))
        del M, S
    A = torch.empty_like(A0)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    recs = []
    seen = set()
    for outer, inner in grid:
        o, i = min(outer, n), min(inner, outer, n)
        if (o, i) in seen:
            continue
        seen.add((o, i))

        def run(o=o, i=i):
            A.copy_(A0)
            if op == "potrf":
                call("double_blocked_potrf_kblocked_syrk", handle.ptr, P(A.data_ptr()), n, n, o,
                     i, 0, P(info.data_ptr()))
            else:
                call("double_blocked_getrf", handle.ptr, P(A.data_ptr()), n, n, o, i, 0, 0,
                     P(ipiv.data_ptr()), P(info.data_ptr()))
        ms = _time(torch, run, reps)
        recs.append({"op": op, "n": n, "outer": o, "inner": i, "ms": ms})
    del A, A0
    return recs


def _matrix(torch, handle, op, n, seed):
    """Timing input: general U[-1,1) or the symmetric diagonally dominant
    (A + A^T)/2 + n I (SPD by Gershgorin), both FP32 on the device."""
    P = ctypes.c_void_p
    A = torch.empty(n * n, dtype=torch.float32, device="cuda")
    lib().hdbf_fill_uniform(handle.ptr, P(A.data_ptr()), n * n, seed, 0)
    if op == "potrf":
        M = A.view(n, n)
        M.add_(M.t().clone()).mul_(0.5)
        M.diagonal().add_(float(n))
    return A


def time_candidates(torch, handle, op, precision, n, A0, reps=1):
    """{selector class index: ms} for one (op, precision, n); candidates that
    clamp to the same effective configuration share one measurement."""
    from .selector import CANDIDATES, candidate_kind
    P = ctypes.c_void_p
    kind = candidate_kind(op, precision)
    A = torch.empty_like(A0)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    done, out = {}, {}
    for k, (ck, par) in enumerate(CANDIDATES):
        if ck != kind:
            continue
        if kind == "blocks":
            o = min(par[0], n)
            key = (o, min(par[1], o))
        else:
            key = (min(par[0], n),)
        if key not in done:
            def run(key=key):
                A.copy_(A0)
                if kind == "blocks" and op == "potrf":
                    call("double_blocked_potrf_kblocked_syrk", handle.ptr, P(A.data_ptr()), n, n,
                         key[0], key[1], 0, P(info.data_ptr()))
                elif kind == "blocks":
                    call("double_blocked_getrf", handle.ptr, P(A.data_ptr()), n, n, key[0], key[1],
                         0, 0, P(ipiv.data_ptr()), P(info.data_ptr()))
                elif op == "potrf":
                    lib().hdbf_spotrf_mixed(handle.ptr, PREC[precision], P(A.data_ptr()), n, n,
                                            key[0], P(info.data_ptr()))
                else:
                    lib().hdbf_sgetrf_mixed(handle.ptr, PREC[precision], P(A.data_ptr()), n, n,
                                            key[0], P(ipiv.data_ptr()), P(info.data_ptr()))
            done[key] = _time(torch, run, reps)
        out[k] = done[key]
    del A
    return out


def random_mix(rng, heldout=False):
    """A random uneven batch: counts and order ranges around the 4096 SPD
    n~U[16,512] / 2048 general n~U[32,768] workload.  Held-out mixes come
    from a different family (one narrow order band per operation)."""
    if not heldout:
        n_spd = int(rng.integers(0, 4097))
        n_gen = int(rng.integers(0 if n_spd >= 16 else 16, 2049))
        lo_s = int(rng.integers(16, 129)); hi_s = int(rng.integers(lo_s + 16, 513))
        lo_g = int(rng.integers(32, 257)); hi_g = int(rng.integers(lo_g + 32, 769))
    else:
        n_spd = int(rng.integers(256, 3073))
        n_gen = int(rng.integers(128, 1537))
        c_s = int(rng.integers(48, 481)); c_g = int(rng.integers(64, 705))
        lo_s, hi_s = max(16, c_s - 32), min(512, c_s + 32)
        lo_g, hi_g = max(32, c_g - 64), min(768, c_g + 64)
    ns = np.concatenate([rng.integers(lo_s, hi_s + 1, size=n_spd),
                         rng.integers(lo_g, hi_g + 1, size=n_gen)]).astype(np.int32)
    ops = np.concatenate([np.zeros(n_spd, np.int32), np.ones(n_gen, np.int32)])
    return ops, ns


def collect(torch, handle, nmax=32768, step=1024, mixes=48, heldout_mixes=16, seed=4,
            log=None):
    """Selector records over the tuning grid (see the module docstring)."""
    recs = []
    orders = sorted(set(list(range(step, nmax + 1, step)) +
                        list(range(step + step // 2, nmax, step))))
    for n in orders:
        for op in ("potrf", "getrf"):
            A0 = _matrix(torch, handle, op, n, seed + n)
            for prec in ("fp32", "bf16", "fp16"):
                t = time_candidates(torch, handle, op, prec, n, A0)
                recs.append({"op": op, "precision": prec, "ns": [n],
                             "times": {str(k): v for k, v in t.items()}})
                if log:
                    log(op, prec, n, {k: round(v, 3) for k, v in t.items()})
            del A0
            torch.cuda.empty_cache()
    rng = np.random.default_rng(seed)
    for i in range(mixes + heldout_mixes):
        held = i >= mixes
        ops, ns = random_mix(rng, held)
        b = batch_mod.DeviceBatch(torch, ops, ns)
        batch_mod.fill_batch(torch, handle, b, seed + i)
        _, res = tune_batched(torch, handle, b, reps=1)
        # the selector's batched candidates are the variants it names
        cls = {c[1][0]: k for k, c in enumerate(_candidates()) if c[0] == "variant"}
        from .selector import order_stats
        recs.append({"op": "batched", "precision": "fp32", "stats": order_stats(ns),
                     "lu_fraction": float(ops.mean()), "heldout": held,
                     "times": {str(cls[v]): ms for v, ms in res.items() if v in cls}})
        if log:
            log("batched", len(ns), held, {v: round(ms, 3) for v, ms in res.items()})
        del b
    return recs


def _candidates():
    from .selector import CANDIDATES
    return CANDIDATES
