"""Exhaustive autotuner.

* ``tune_batched`` times every CTA-size variant of the persistent batched
  kernel on a batch (inputs restored before each timed run) and returns the
  fastest.
* ``tune_blocks`` times a grid of (outer block, inner block) choices for the
  large double-blocked factorizations at one order n and returns the fastest;
  its records are the training data of the learned selector
  (``hygondoubleblockedfactorizations_b200.selector``).
Timings are CUDA-event device times after a warm-up run (the warm-up also
records the CUDA graph the library replays).
"""
from __future__ import annotations

import ctypes

from . import batch as batch_mod
from . import call, lib


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
