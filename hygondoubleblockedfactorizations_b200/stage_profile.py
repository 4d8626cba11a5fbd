"""Per-stage profile of one factorization (the role of the reference's
``profile_double_blocked_potrf`` / ``profile_double_blocked_getrf``
executables, src/potrf/benchmark/profile_double_blocked_potrf.cpp and
src/getrf/benchmark/profile_double_blocked_getrf.cpp).

    python -m hygondoubleblockedfactorizations_b200.stage_profile \\
        --op getrf --precision fp32 --n 8192 --outer 8192 --inner 512 [--reps 1]

Builds the seeded input on the device (POTRF: (A + A^T)/2 + n I from the
counter-based U[-1,1) stream; GETRF: U[-1,1)), runs one warm-up call (which
also records the call's profiled CUDA graph), then ``reps`` profiled calls, and prints
one JSON line: total time, TFLOP/s (n^3/3 or 2n^3/3) and, per kernel class,
launches, milliseconds, share of the device time and TFLOP/s or GB/s.
``--stage-samples`` adds the reference's stage tables
(src/getrf/profile_double_blocked_getrf.cpp, src/potrf/profile_double_blocked_potrf.cpp):
for each of the ``--reps`` profiled calls a ``STAGE_SAMPLE <OP> iteration=<i>``
table of the driver's stages (Stage | Total(ms) | Calls | Avg(ms) | Share |
GFLOPS, the layout of include/utils/benchmark/stage_breakdown_profiler.h:91-130),
then the spread of each stage and of the total over the samples (mean, sample
standard deviation, relative standard deviation in percent, minimum and
maximum, as the reference's stage-spread statistics).
``--panel`` selects the GETRF panel kernel (0 automatic, 1 grid-wide,
2 cluster); ``--batched`` runs the FP32 GETRF through
``double_blocked_getrf_batched_pivot`` (iterative outer TRSM, as the
benchmark does) instead of ``double_blocked_getrf``, and ``--lookahead 0|1``
sets the handle's GETRF look-ahead.  Mixed precisions use ``hdbf_spotrf_mixed`` / ``hdbf_sgetrf_mixed``
with panel width ``--inner``; ``--precision fp64`` runs the FP64 twins
``double_blocked_potrf_double`` / ``double_blocked_getrf_double`` (iterative
outer TRSM) on the same inputs widened to FP64.
"""
from __future__ import annotations

import argparse
import ctypes
import json


def main(argv=None):
    import torch

    from . import PREC, Handle, call, lib
    from .tuner import _matrix

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--op", choices=["potrf", "getrf", "posv", "gesv", "batched"],
                    default="getrf")
    ap.add_argument("--precision", choices=list(PREC) + ["fp64"], default="fp32")
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--outer", type=int, default=8192)
    ap.add_argument("--inner", type=int, default=512)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--panel", type=int, default=None)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--batched", action="store_true")
    ap.add_argument("--lookahead", type=int, default=None)
    ap.add_argument("--stage-samples", action="store_true")
    ap.add_argument("--trsm-block", type=int, default=0,
                    help="GETRF --batched: row block of the iterative outer TRSM (0: direct)")
    ap.add_argument("--syrk-k-tile", type=int, default=0,
                    help="FP32 POTRF: K tile of the outer SYRK (0: the SYRK runs inside the "
                         "outer GEMM launch)")
    a = ap.parse_args(argv)

    P = ctypes.c_void_p
    if a.op in ("posv", "gesv", "batched"):
        return solve_driver(torch, a)
    h = Handle(torch.cuda.current_stream().cuda_stream)
    if a.panel is not None:
        h.set_panel_kernel(a.panel)
    if a.lookahead is not None:
        h.set_lookahead(bool(a.lookahead))
    n = a.n
    A0 = _matrix(torch, h, a.op, n, a.seed)
    if a.precision == "fp64":
        A0 = A0.double()
    A = torch.empty_like(A0)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    if a.batched:
        import numpy as np

        from . import WorkspacePivot
        tile = 64
        keep = [torch.zeros(n, dtype=torch.int32, device="cuda"),
                torch.zeros(n, dtype=torch.int32, device="cuda"),
                torch.zeros(n * tile, dtype=torch.float32, device="cuda")]
        host = [np.zeros(n, np.int32) for _ in range(4)]
        ws = WorkspacePivot(keep[0].data_ptr(), keep[1].data_ptr(), keep[2].data_ptr(),
                            *[x.ctypes.data for x in host], n, tile)

    def run():
        A.copy_(A0)
        if a.precision == "fp64" and a.op == "potrf":
            call("double_blocked_potrf_double", h.ptr, P(A.data_ptr()), n, n, a.outer, a.inner,
                 P(info.data_ptr()))
        elif a.precision == "fp64":
            call("double_blocked_getrf_double", h.ptr, P(A.data_ptr()), n, n, a.outer, a.inner,
                 1, 0, P(ipiv.data_ptr()), P(info.data_ptr()))
        elif a.precision == "fp32" and a.op == "potrf":
            call("double_blocked_potrf_kblocked_syrk", h.ptr, P(A.data_ptr()), n, n, a.outer,
                 a.inner, a.syrk_k_tile, P(info.data_ptr()))
        elif a.precision == "fp32" and a.batched:
            call("double_blocked_getrf_batched_pivot", h.ptr, P(A.data_ptr()), n, n, a.outer,
                 a.inner, 1, a.trsm_block, 0, P(ipiv.data_ptr()), P(info.data_ptr()),
                 ctypes.byref(ws))
        elif a.precision == "fp32":
            call("double_blocked_getrf", h.ptr, P(A.data_ptr()), n, n, a.outer, a.inner, 0, 0,
                 P(ipiv.data_ptr()), P(info.data_ptr()))
        elif a.op == "potrf":
            st = lib().hdbf_spotrf_mixed(h.ptr, PREC[a.precision], P(A.data_ptr()), n, n, a.inner,
                                         P(info.data_ptr()))
            assert st == 0, st
        else:
            st = lib().hdbf_sgetrf_mixed(h.ptr, PREC[a.precision], P(A.data_ptr()), n, n, a.inner,
                                         P(ipiv.data_ptr()), P(info.data_ptr()))
            assert st == 0, st

    # warm-up with the profiler on: records the profiled CUDA graph replayed below
    h.profile_begin()
    run()
    torch.cuda.synchronize()
    h.profile_end()
    h.check("warm-up")
    samples = []
    if a.stage_samples:
        for it in range(a.reps):
            h.profile_begin()
            run()
            torch.cuda.synchronize()
            h.profile_end()
            samples.append(h.profile_stages())
            print_stage_sample(a.op.upper(), it + 1, samples[-1])
        print_spread(samples)
    # wall time of `reps` calls without the profiler, then one profiled call
    # for the per-class split (a profiled graph replay keeps one replay's times)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    h.profile_begin()
    run()
    torch.cuda.synchronize()
    prof = h.profile_end()
    flops = n ** 3 / 3.0 if a.op == "potrf" else 2.0 * n ** 3 / 3.0
    dev_ms = sum(v[1] for v in prof.values())
    stages = {}
    for k, (nl, t, fl, by) in sorted(prof.items(), key=lambda kv: -kv[1][1]):
        stages[k] = {"launches": nl, "ms": round(t, 3),
                     "share": round(t / dev_ms, 4) if dev_ms else None,
                     "tflops": round(fl / (t / 1e3) / 1e12, 3) if fl and t else None,
                     "gbs": round(by / (t / 1e3) / 1e9, 1) if by and t else None}
    out = {"op": a.op, "precision": a.precision, "n": n, "outer": a.outer, "inner": a.inner,
           "panel": a.panel, "batched": a.batched, "lookahead": a.lookahead, "ms": round(ms, 3), "tflops": round(flops / (ms / 1e3) / 1e12, 3),
           "info": int(info.item()), "device_errors": h.device_errors(), "stages": stages}
    if samples:
        out["stage_spread"] = spread(samples)
    print(json.dumps(out), flush=True)
    return out


def solve_driver(torch, a):
    """--op posv / gesv: one mixed-precision (or FP32) factorization plus FP64
    classical refinement (hdbf_dposv_mixed / hdbf_dgesv_mixed, nrhs 16) on an
    SPD / general matrix with eigen- / singular values log-spaced in [1, 1e2];
    --op batched: the uneven batched factor-and-solve launch on a batch of
    --n systems (SPD n ~ U[16, 512] and general n ~ U[32, 768], half each).
    Runs --reps calls after one warm-up and prints the per-class profile."""
    import ctypes

    from . import PREC, Handle, IrInfo, call
    from . import batch as bm
    P = ctypes.c_void_p
    h = Handle(torch.cuda.current_stream().cuda_stream)
    if a.op == "batched":
        ops, ns = bm.config3_sizes(n_spd=a.n // 2, n_gen=a.n - a.n // 2)
        b = bm.DeviceBatch(torch, ops, ns)
        bm.fill_batch(torch, h, b, 3)

        def run():
            bm.restore(b)
            assert b.run(h, 2) == 0
    else:
        n, nrhs = a.n, 16
        g = torch.Generator(device="cuda")
        g.manual_seed(a.seed)
        Q, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
        lam = torch.logspace(0.0, 2.0, n, dtype=torch.float64, device="cuda")
        if a.op == "posv":
            A = (Q * lam) @ Q.t()
            A = 0.5 * (A + A.t())
        else:
            V, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda",
                                               generator=g))
            A = (Q * lam) @ V.t()
        A = A.t().contiguous()
        B = torch.randn(nrhs, n, dtype=torch.float64, device="cuda", generator=g)
        X = torch.zeros_like(B)
        fn = "hdbf_dposv_mixed" if a.op == "posv" else "hdbf_dgesv_mixed"

        def run():
            info = IrInfo()
            st = call(fn, h.ptr, PREC[a.precision], 0, P(A.data_ptr()), n, n, nrhs,
                      P(B.data_ptr()), n, P(X.data_ptr()), n, ctypes.c_double(1e-13), 30,
                      ctypes.byref(info))
            assert st == 0 and info.converged == 1, (st, info.backward_error)
    for _ in range(max(1, a.reps)):  # warm-up (records the graphs)
        run()
    torch.cuda.synchronize()
    h.profile_begin()
    run()
    torch.cuda.synchronize()
    prof = h.profile_end()
    out = {"op": a.op, "precision": a.precision, "n": a.n,
           "kernels": {k: {"launches": v[0], "ms": round(v[1], 3)}
                       for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])}}
    print(json.dumps(out), flush=True)
    h.close()
    return out


def print_stage_sample(op, iteration, stages, width=110):
    """One STAGE_SAMPLE table (stage_breakdown_profiler.h:91-130 layout)."""
    print("=" * width)
    print(f"STAGE_SAMPLE {op} iteration={iteration}")
    print("=" * width)
    print(f"{'Stage':24s} | {'Total(ms)':>12s} | {'Calls':>10s} | {'Avg(ms)':>12s} | "
          f"{'Share':>10s} | {'GFLOPS':>12s}")
    print("-" * width)
    total = sum(v[1] for v in stages.values())
    for name, (calls, t, fl) in stages.items():
        share = 100.0 * t / total if total > 0 else 0.0
        gf = fl / (t / 1e3) / 1e9 if t > 0 else 0.0
        print(f"{name:24s} | {t:12.3f} | {calls:10d} | {t / max(calls, 1):12.3f} | "
              f"{share:9.2f}% | {gf:12.2f}")
    print("=" * width)


def spread(samples):
    """Per stage and for the total: mean, sample SD, RSD %, min, max (ms)."""
    import statistics
    names = list(dict.fromkeys(k for smp in samples for k in smp))
    out = {}
    for name in names + ["Total"]:
        vals = [sum(v[1] for v in smp.values()) if name == "Total" else smp.get(name, (0, 0.0, 0))[1]
                for smp in samples]
        mean = statistics.mean(vals)
        sd = statistics.stdev(vals) if len(vals) > 1 else 0.0
        out[name] = {"mean_ms": round(mean, 4), "sample_sd_ms": round(sd, 4),
                     "rsd_percent": round(100.0 * sd / mean, 4) if mean > 0 else 0.0,
                     "min_ms": round(min(vals), 4), "max_ms": round(max(vals), 4)}
    return out


def print_spread(samples):
    print(f"{'stage':24s},mean_ms,sample_sd_ms,rsd_percent,min_ms,max_ms")
    for name, st in spread(samples).items():
        print(f"{name:24s},{st['mean_ms']},{st['sample_sd_ms']},{st['rsd_percent']},"
              f"{st['min_ms']},{st['max_ms']}")


if __name__ == "__main__":
    main()
