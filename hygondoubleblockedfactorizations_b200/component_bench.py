"""Component benchmarks of the SYRK, TRSM and GEMM families, with the
reference's CSV schema (the role of its ``benchmark_syrk`` / ``benchmark_trsm``
/ ``benchmark_gemm`` executables: src/syrk/test_syrk.cpp:6-54,
src/trsm/test_trsm.cpp:15-85, src/gemm/gemm_benchmark.cpp:215-357).

    python -m hygondoubleblockedfactorizations_b200.component_bench syrk N K [ERROR_MODE]
        [--nb NB ...] [--k-tile TK ...]
    python -m hygondoubleblockedfactorizations_b200.component_bench trsm N M [ERROR_MODE]
        [--nb NB ...] [--double-nb NB ...] [--b B ...]
    python -m hygondoubleblockedfactorizations_b200.component_bench gemm [K]
    python -m hygondoubleblockedfactorizations_b200.component_bench gemm --shape M N K
        [--m-tile TM]

ERROR_MODE as the reference's (utils/benchmark/error_mode.h): 0 none,
1 forward error, 2 sampled relative residual, 3 both.  Iterations come from
BENCHMARK_WARMUP_ITERS (default 2) and BENCHMARK_PROFILE_ITERS (default 5);
each timed iteration restores the output operand first (outside the timed
interval) and is timed alone with CUDA events on the handle's stream.  When
BENCHMARK_CSV_PATH is set, one row per timed iteration is written there with
the reference's columns (src/utils/benchmark/benchmark_printer.cpp:26-68):

    benchmark,method,parameters,iteration,time_ms,mean_ms,median_ms,stddev_ms,
    min_ms,max_ms,gflops,speedup,forward_error,residual_metric,residual_value

Operations and flop counts follow the reference's cases:
* SYRK  C(lower) -= A A^T, A n x k, C n x n; n (n + 1) k flops.  Methods:
  this library's single-call SYRK (the baseline, in place of rocBLAS ssyrk),
  K-blocked per --k-tile, recursive (nb), bottom-up batched (nb) and the
  mixed-precision batched SYRK (FP16 tensor cores).
* TRSM  B (n x m) <- B L^{-T}, L m x m lower; n m^2 flops.  Methods: the
  single-call TRSM (baseline), recursive (nb), recursive with tiled update,
  iterative right-looking (nb), double-blocked (nb x b), mixed recursive.
* GEMM  C -= A B^T (this library's NT update): the right-looking Cholesky
  shapes of the reference (M = N = 32768 - K for each K step) or one explicit
  shape, optionally M-tiled; 2 M N K flops.
Forward errors are against an FP64 product on the device (torch, outside the
timed region); sampled residuals recompute 4096 random entries in FP64 on the
host, as the reference's verify_sampled_relative_residual does.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import statistics
import sys

import numpy as np

from . import Handle, call, lib

P = ctypes.c_void_p
CSV_HEADER = ("benchmark,method,parameters,iteration,time_ms,mean_ms,median_ms,stddev_ms,"
              "min_ms,max_ms,gflops,speedup,forward_error,residual_metric,residual_value")


def _iters():
    warm = max(0, int(os.environ.get("BENCHMARK_WARMUP_ITERS", "2")))
    iters = max(1, int(os.environ.get("BENCHMARK_PROFILE_ITERS", "5")))
    return warm, iters


class Runner:
    """Times each method, keeps the reference's BenchmarkResult fields."""

    def __init__(self, torch, title, flops, error_mode, residual_metric):
        self.torch, self.title, self.flops = torch, title, flops
        self.error_mode, self.metric = error_mode, residual_metric
        self.results = []
        self.baseline = None

    def run(self, method, params, reset, fn, verify):
        torch = self.torch
        warm, iters = _iters()
        for _ in range(warm):
            reset()
            fn()
        torch.cuda.synchronize()
        times = []
        for _ in range(iters):
            reset()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        mean = sum(times) / len(times)
        fwd, res = verify() if self.error_mode else (-1.0, -1.0)
        if self.baseline is None:
            self.baseline = mean
        r = {"method": method, "parameters": params, "times": times, "mean": mean,
             "median": statistics.median(times),
             "stddev": statistics.pstdev(times) if len(times) > 1 else 0.0,
             "min": min(times), "max": max(times),
             "gflops": self.flops / (mean / 1e3) / 1e9 if mean > 0 else 0.0,
             "speedup": self.baseline / mean if mean > 0 else 0.0,
             "forward_error": fwd, "residual_value": res}
        self.results.append(r)
        return r

    def report(self):
        show_res = self.error_mode in (2, 3)
        show_fwd = self.error_mode in (1, 3)
        print(f"\n{self.title}")
        head = f"{'Method':32s} | {'Parameters':14s} | {'Time(ms)':>10s} | {'GFLOPS':>10s} | {'Speedup':>7s}"
        if show_fwd:
            head += f" | {'Forward Error':>13s}"
        if show_res:
            head += f" | {'Sampled Rel. Residual':>21s}"
        print(head)
        for r in self.results:
            line = (f"{r['method']:32s} | {r['parameters']:14s} | {r['mean']:10.3f} | "
                    f"{r['gflops']:10.1f} | {r['speedup']:7.2f}")
            if show_fwd:
                line += f" | {r['forward_error']:13.3e}"
            if show_res:
                line += f" | {r['residual_value']:21.3e}"
            print(line)
        path = os.environ.get("BENCHMARK_CSV_PATH")
        if path:
            metric = self.metric if show_res else "none"
            q = lambda s: '"' + str(s).replace('"', '""') + '"'  # noqa: E731
            with open(path, "w") as f:
                f.write(CSV_HEADER + "\n")
                for r in self.results:
                    for i, t in enumerate(r["times"]):
                        f.write(",".join([q(self.title), q(r["method"]), q(r["parameters"]), str(i),
                                          repr(t), repr(r["mean"]), repr(r["median"]),
                                          repr(r["stddev"]), repr(r["min"]), repr(r["max"]),
                                          repr(r["gflops"]), repr(r["speedup"]),
                                          repr(r["forward_error"]), metric,
                                          repr(r["residual_value"])]) + "\n")
            print(f"Raw timing CSV: {path}")


def _uniform(torch, h, count, seed):
    x = torch.empty(count, dtype=torch.float32, device="cuda")
    st = lib().hdbf_fill_uniform(h.ptr, P(x.data_ptr()), count, seed, 0)
    assert st == 0
    return x


def _rel_fro(ref, got):
    d = (ref - got).double()
    return float(d.norm() / max(float(ref.double().norm()), 1e-300))


def _samples(rows, cols, count, lower=False, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        r, c = int(rng.integers(0, rows)), int(rng.integers(0, cols))
        if lower and r < c:
            continue
        out.append((r, c))
    return out


def bench_syrk(torch, a):
    n, k = a.n, a.k
    h = Handle(torch.cuda.current_stream().cuda_stream)
    pool = ctypes.c_void_p()
    lib().hdbf_stream_pool_create(16, ctypes.byref(pool))
    A = _uniform(torch, h, n * k, 3)                       # column-major n x k, lda = n
    C0 = _uniform(torch, h, n * n, 4)                      # column-major n x n
    C = torch.empty_like(C0)
    flops = float(n) * (n + 1) * k
    Am = A.view(k, n).t()                                  # n x k matrix view
    gold = None
    if a.error_mode in (1, 3):
        Cd = C0.view(n, n).t().double()
        gold = torch.tril(Cd - Am.double() @ Am.double().t())
    Ah = A.cpu().numpy().reshape(k, n).T
    C0h = C0.cpu().numpy().reshape(n, n).T

    def verify():
        fwd = res = -1.0
        Cm = C.view(n, n).t()
        if gold is not None:
            fwd = _rel_fro(gold, torch.tril(Cm.double()))
        if a.error_mode in (2, 3):
            Ch = C.cpu().numpy().reshape(n, n).T
            num = den = 0.0
            for r, c in _samples(n, n, 4096, lower=True):
                ref = float(C0h[r, c]) - float(np.dot(Ah[r].astype(np.float64), Ah[c].astype(np.float64)))
                num += (float(Ch[r, c]) - ref) ** 2
                den += ref * ref
            res = (num ** 0.5) / (den ** 0.5 + 1e-20)
        return fwd, res

    run = Runner(torch, f"SYRK benchmark: C(lower) -= A A^T, N={n} K={k}", flops, a.error_mode,
                 "sampled_relative_residual")
    reset = lambda: C.copy_(C0)  # noqa: E731
    run.run("Single call (FP32)", "N/A", reset,
            lambda: call("syrk_lower_update", h.ptr, n, k, P(A.data_ptr()), n, P(C.data_ptr()), n),
            verify)
    for tk in a.k_tile:
        run.run("K-blocked (FP32)", f"tk={tk}", reset,
                lambda tk=tk: call("syrk_lower_update_kblocked", h.ptr, n, k, P(A.data_ptr()), n,
                                   P(C.data_ptr()), n, tk), verify)
    for nb in a.nb:
        run.run("Recursive (FP32)", f"nb={nb}", reset,
                lambda nb=nb: call("recursive_syrk_parallel", h.ptr, P(A.data_ptr()), n,
                                   P(C.data_ptr()), n, n, k, nb), verify)
        run.run("Batched (FP32)", f"nb={nb}", reset,
                lambda nb=nb: call("batched_syrk_bottom_up", h.ptr, pool, P(A.data_ptr()), n,
                                   P(C.data_ptr()), n, n, k, nb), verify)
        run.run("Batched (Mixed)", f"nb={nb}", reset,
                lambda nb=nb: call("batched_syrk_bottom_up_mixed", h.ptr, pool, P(A.data_ptr()),
                                   n, P(C.data_ptr()), n, n, k, nb), verify)
    h.check("syrk")
    run.report()
    lib().hdbf_stream_pool_destroy(pool)
    h.close()
    return run.results


def bench_trsm(torch, a):
    n, m = a.n, a.m
    h = Handle(torch.cuda.current_stream().cuda_stream)
    # L: m x m lower with U[-1,1) entries and a dominant diagonal (m + |g|),
    # so the solve is well conditioned at every m; B: n x m U[-1,1)
    G = _uniform(torch, h, m * m, 5).view(m, m).t()
    Lm = torch.tril(G)
    Lm.diagonal().copy_(float(m) + G.diagonal().abs())
    L = Lm.t().contiguous().view(-1)                       # column-major storage
    B0 = _uniform(torch, h, n * m, 6)
    B = torch.empty_like(B0)
    flops = float(n) * m * m
    gold = None
    if a.error_mode in (1, 3):
        Bd = B0.view(m, n).t().double()
        gold = torch.linalg.solve_triangular(Lm.double(), Bd.t(), upper=False).t()
    Lh = L.cpu().numpy().reshape(m, m).T
    B0h = B0.cpu().numpy().reshape(m, n).T

    def verify():
        fwd = res = -1.0
        X = B.view(m, n).t()
        if gold is not None:
            fwd = _rel_fro(gold, X.double())
        if a.error_mode in (2, 3):
            Xh = B.cpu().numpy().reshape(m, n).T
            num = den = 0.0
            for r, c in _samples(n, m, 4096):
                rec = float(np.dot(Xh[r, :c + 1].astype(np.float64), Lh[c, :c + 1].astype(np.float64)))
                ref = float(B0h[r, c])
                num += (rec - ref) ** 2
                den += ref * ref
            res = (num ** 0.5) / (den ** 0.5 + 1e-20)
        return fwd, res

    run = Runner(torch, f"TRSM benchmark: B <- B L^-T, N={n} M={m}", flops, a.error_mode,
                 "sampled_relative_residual")
    reset = lambda: B.copy_(B0)  # noqa: E731
    run.run("Single call (FP32)", "N/A", reset,
            lambda: call("trsm_right_lower_transpose", h.ptr, n, m, P(L.data_ptr()), m,
                         P(B.data_ptr()), n), verify)
    for nb in a.nb:
        run.run("Recursive (FP32)", f"nb={nb}", reset,
                lambda nb=nb: call("recursive_trsm", h.ptr, P(L.data_ptr()), m, P(B.data_ptr()),
                                   n, n, m, nb), verify)
        run.run("Recursive tiled update (FP32)", f"nb={nb}", reset,
                lambda nb=nb: call("recursive_trsm_tiled_update", h.ptr, P(L.data_ptr()), m,
                                   P(B.data_ptr()), n, n, m, nb), verify)
        run.run("Iterative right-looking (FP32)", f"nb={nb}", reset,
                lambda nb=nb: call("iterative_trsm_right_looking", h.ptr, P(L.data_ptr()), m,
                                   P(B.data_ptr()), n, n, m, nb), verify)
        run.run("Recursive (Mixed)", f"nb={nb}", reset,
                lambda nb=nb: call("recursive_trsm_mixed", h.ptr, P(L.data_ptr()), m,
                                   P(B.data_ptr()), n, n, m, nb), verify)
    for dnb in a.double_nb:
        for b in (a.b or [256]):
            run.run("Double-blocked (FP32)", f"nb={dnb},b={b}", reset,
                    lambda dnb=dnb, b=b: call("double_blocked_trsm", h.ptr, P(L.data_ptr()), m,
                                              P(B.data_ptr()), n, n, m, dnb, b), verify)
    h.check("trsm")
    run.report()
    h.close()
    return run.results


def bench_gemm(torch, a):
    h = Handle(torch.cuda.current_stream().cuda_stream)
    if a.shape:
        shapes = [tuple(a.shape)]
    else:
        total = 32768
        ks = [a.k_step] if a.k_step else [64, 128, 256, 384, 512, 768, 1024, 1536, 2048, 3072,
                                           4096, 6144, 8192, 12288, 16384]
        shapes = [(total - k, total - k, k) for k in ks]
    all_res = []
    for M, N, K in shapes:
        A = _uniform(torch, h, M * K, 7)
        Bm = _uniform(torch, h, N * K, 8)
        C0 = _uniform(torch, h, M * N, 9)
        C = torch.empty_like(C0)
        gold = None
        if a.error_mode in (1, 3):
            gold = (C0.view(N, M).t().double()
                    - A.view(K, M).t().double() @ Bm.view(K, N).t().double().t())
        Ah = Bh = C0h = None
        if a.error_mode in (2, 3):
            Ah = A.cpu().numpy().reshape(K, M).T
            Bh = Bm.cpu().numpy().reshape(K, N).T
            C0h = C0.cpu().numpy().reshape(N, M).T

        def verify():
            fwd = res = -1.0
            if gold is not None:
                fwd = _rel_fro(gold, C.view(N, M).t().double())
            if Ah is not None:
                Ch = C.cpu().numpy().reshape(N, M).T
                num = den = 0.0
                for r, c in _samples(M, N, 4096):
                    ref = float(C0h[r, c]) - float(np.dot(Ah[r].astype(np.float64),
                                                          Bh[c].astype(np.float64)))
                    num += (float(Ch[r, c]) - ref) ** 2
                    den += ref * ref
                res = (num ** 0.5) / (den ** 0.5 + 1e-20)
            return fwd, res

        run = Runner(torch, f"GEMM benchmark: C -= A B^T, M={M} N={N} K={K}", 2.0 * M * N * K,
                     a.error_mode, "sampled_relative_residual")
        reset = lambda: C.copy_(C0)  # noqa: E731
        run.run("NT update (FP32)", "N/A", reset,
                lambda: call("gemm_nt_update", h.ptr, M, N, K, P(A.data_ptr()), M,
                             P(Bm.data_ptr()), N, P(C.data_ptr()), M), verify)
        if a.m_tile:
            run.run("NT update M-tiled (FP32)", f"m_tile={a.m_tile}", reset,
                    lambda: call("gemm_nt_update_m_tiled", h.ptr, M, N, K, P(A.data_ptr()), M,
                                 P(Bm.data_ptr()), N, P(C.data_ptr()), M, a.m_tile), verify)
        run.report()
        all_res.extend(run.results)
        del A, Bm, C0, C, gold
        torch.cuda.empty_cache()
    h.check("gemm")
    h.close()
    return all_res


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="family", required=True)
    s = sub.add_parser("syrk")
    s.add_argument("n", type=int)
    s.add_argument("k", type=int)
    s.add_argument("error_mode", type=int, nargs="?", default=0)
    s.add_argument("--nb", type=int, nargs="*", default=[256])
    s.add_argument("--k-tile", type=int, nargs="*", default=[])
    t = sub.add_parser("trsm")
    t.add_argument("n", type=int)
    t.add_argument("m", type=int)
    t.add_argument("error_mode", type=int, nargs="?", default=0)
    t.add_argument("--nb", type=int, nargs="*", default=[256])
    t.add_argument("--double-nb", type=int, nargs="*", default=[])
    t.add_argument("--b", type=int, nargs="*", default=[])
    g = sub.add_parser("gemm")
    g.add_argument("k_step", type=int, nargs="?", default=None)
    g.add_argument("--shape", type=int, nargs=3, metavar=("M", "N", "K"))
    g.add_argument("--m-tile", type=int, default=0)
    g.add_argument("--error-mode", type=int, default=0)
    a = ap.parse_args(argv)
    if a.family == "syrk":
        return bench_syrk(torch, a)
    if a.family == "trsm":
        return bench_trsm(torch, a)
    return bench_gemm(torch, a)


if __name__ == "__main__":
    main(sys.argv[1:])
