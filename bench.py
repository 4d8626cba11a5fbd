"""Benchmark: POTRF + GETRF TFLOP/s at n = 32768 on one B200 (FP32 path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n 32768] [--impl ours|reference]

Workload (per step, per rank): one double-blocked Cholesky of the SPD matrix
A = G G^T / n + I (G iid U[-1,1) FP32, seed 0, formed in FP64, rounded to FP32)
and one double-blocked partially pivoted LU of an iid U[-1,1) FP32 matrix
(seed 1), n = 32768, column-major, lda = n.  Each step restores both inputs
from pristine device copies (a 4.3 GB device-to-device copy each, included in
the timed step) and factors them in place; inputs are far larger than the
126 MB L2, so no flush is needed.  FLOPs: n^3/3 (POTRF) + 2 n^3/3 (GETRF), the
reference's counting (potrf_benchmark_common.cpp:31, getrf_benchmark_common.cpp:32).

value  = whole-job TFLOP/s with inputs resident in HBM (device-timed, CUDA events,
         max over ranks; multi-GPU runs are independent replicas, weak scaling).
e2e    = the same step through the C ABI starting from pinned HOST buffers:
         H2D of each input, factorization, D2H of the factors, pivots and info.
roofline = the dominant kernel (sgemm_sub_kernel, FP32 SIMT FFMA) from the
         library's per-launch event profiler over the timed region, against the
         FP32 SIMT peak (SMs x 128 lanes x 2 flop x max SM clock).
cpu_baseline = host LAPACK spotrf + sgetrf (SciPy's OpenBLAS, all host threads),
         one step on the bench's own n=32768 inputs; the same leg then checks the
         factors of the last timed step (parity object): CPU FP64 scaled
         residuals <= 10 beside host LAPACK's, pivots vs host sgetrf.  The run
         exits non-zero when that check fails.
--impl reference = host LAPACK spotrf + sgetrf at the same n, all host threads,
         as many full steps as fit in about six minutes (at least one).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "POTRF+GETRF FP32 TFLOP/s at n=32768 (double-blocked, one B200)"
UNIT = "TFLOP/s"


def flops_potrf(n):
    return n ** 3 / 3.0


def flops_getrf(n):
    return 2.0 * n ** 3 / 3.0


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling (every 200 ms) during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.idx), "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        power = [num(r[3]) for r in rows if num(r[3]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        # "under load" = samples at >= 50% of the peak power seen
        pmax = max(power) if power else 0
        loaded = [num(r[1]) for r in rows if num(r[3]) and num(r[3]) >= 0.5 * pmax and num(r[1])]
        return {"sm_mhz": statistics.median(loaded or sm), "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": pmax}


# ----------------------------------------------------------------- CPU LAPACK
def cpu_threads():
    try:
        from threadpoolctl import threadpool_info
        info = [d for d in threadpool_info() if d.get("internal_api") == "openblas"]
        if info:
            return int(info[0]["num_threads"]), info[0].get("version")
    except Exception:
        pass
    return os.cpu_count(), None


def host_inputs(n):
    """The bench's two input families built on the host (the reference arm has
    no device): SPD A = G G^T / n + I with the FP64 product formed by dsyrk
    (the same family as the device's FP64 GEMM; last-bit differences after the
    FP32 rounding are possible), general G iid U[-1,1) (bit-identical)."""
    import oracle  # CPU baseline leg only
    from scipy.linalg import blas
    G0 = oracle.general_uniform(n, 0).astype(np.float64)
    S = blas.dsyrk(1.0 / n, G0, lower=1, trans=0)  # lower triangle of G0 G0^T / n
    del G0
    A = np.empty((n, n), dtype=np.float32, order="F")
    w = 4096
    for j0 in range(0, n, w):  # mirror the lower triangle, add I, round to FP32
        j1 = min(n, j0 + w)
        D = S[j0:j1, j0:j1]
        D = np.tril(D) + np.tril(D, -1).T + np.eye(j1 - j0)
        A[j0:j1, j0:j1] = D
        A[j1:, j0:j1] = S[j1:, j0:j1]
        A[j0:j1, j1:] = S[j1:, j0:j1].T
    del S
    return A, np.asfortranarray(oracle.general_uniform(n, 1))


def lapack_pair(A, G):
    """Host LAPACK spotrf(lower) + sgetrf on copies; returns (L, LU, ipiv, tp, tg)."""
    from scipy.linalg import lapack
    t0 = time.perf_counter()
    c, info = lapack.spotrf(A, lower=1, clean=0, overwrite_a=0)
    t1 = time.perf_counter()
    lu, piv, info2 = lapack.sgetrf(G, overwrite_a=0)
    t2 = time.perf_counter()
    if info != 0 or info2 != 0:
        raise SystemExit(f"host LAPACK failed: spotrf info {info}, sgetrf info {info2}")
    return c, lu, (piv + 1).astype(np.int32), t1 - t0, t2 - t1


def fp64_residual_device(F, A, ipiv):
    """||A - L L^T||_F / ||A||_F (ipiv None; L = lower triangle of F) or
    ||P A - L U||_F / ||A||_F (F packed LU, 1-based LAPACK ipiv), in FP64 with
    torch on the device; F and A are n x n host arrays."""
    import torch
    dev = "cuda"
    n = A.shape[0]
    Fd = torch.from_numpy(np.ascontiguousarray(F.T)).to(dev).double().t()  # F as a matrix
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).to(dev).double().t()
    if ipiv is None:
        L = torch.tril(Fd)
        del Fd
        R = L @ L.t()
        del L
    else:
        L = torch.tril(Fd, -1)
        L.diagonal().fill_(1.0)
        U = torch.triu(Fd)
        del Fd
        R = L @ U
        del L, U
        perm = np.arange(n)
        for r in range(n):
            p = int(ipiv[r]) - 1
            perm[r], perm[p] = perm[p], perm[r]
        Ad = Ad[torch.from_numpy(perm).to(dev)]
    R.sub_(Ad)
    res = float(torch.linalg.matrix_norm(R) / torch.linalg.matrix_norm(Ad))
    del R, Ad
    torch.cuda.empty_cache()
    return res


def cpu_baseline_and_check(n, A, G, gpu):
    """CPU baseline at the bench's own size, and the check of the timed factors.

    Host LAPACK spotrf + sgetrf (SciPy's OpenBLAS, all host threads) run once
    on the SAME FP32 inputs the GPU factored (copied from the device), timed
    with the wall clock around each LAPACK call.  Then the oracle checks the
    GPU's factors from the last timed step against the bound of the
    reference's verify step (potrf_benchmark_common.cpp:294-344,
    getrf_benchmark_common.cpp:54-72): the scaled CPU FP64 residual
    ||A - LL^T||_F / (||A||_F n eps32) and ||PA - LU||_F / (||A||_F n eps32)
    <= 10, beside host LAPACK's own residual on the same input (that one with
    torch's FP64 GEMM on the device, for comparison only), and the GPU
    pivot sequence against sgetrf's (identical, or a first divergence at an
    FP32 near-tie: the two candidates' |s| differ by < 1e-4 relative)."""
    import oracle  # checker and CPU baseline leg only
    thr, ver = cpu_threads()
    Lh, LUh, pivh, tp, tg = lapack_pair(A, G)
    value = (flops_potrf(n) + flops_getrf(n)) / (tp + tg) / 1e12
    base = {"value": round(value, 4), "unit": UNIT, "cores": thr, "kind": "port",
            "sample": (f"host LAPACK spotrf(lower)+sgetrf (SciPy OpenBLAS {ver}, {thr} threads, "
                       f"{os.cpu_count()} host CPUs) on the bench's own n={n} inputs (copied "
                       "from the device), 1 step"),
            "n": n, "potrf_tflops": round(flops_potrf(n) / tp / 1e12, 4),
            "getrf_tflops": round(flops_getrf(n) / tg / 1e12, 4),
            "ms_per_step": round(1e3 * (tp + tg), 1)}
    t0 = time.perf_counter()
    rp_gpu = oracle.scaled(oracle.potrf_residual_tiled(gpu["L"], A), n)
    rg_gpu = oracle.scaled(oracle.getrf_residual_tiled(gpu["LU"], G, gpu["ipiv"]), n)
    # host LAPACK's own residuals, for comparison only: the same FP64 formula
    # evaluated with torch's FP64 GEMM on the device (seconds, not minutes)
    rp_cpu = fp64_residual_device(Lh, A, None) / (n * 2.0 ** -23)
    del Lh
    rg_cpu = fp64_residual_device(LUh, G, pivh) / (n * 2.0 ** -23)
    del LUh
    pv = oracle.pivot_agreement(G, pivh, gpu["ipiv"])
    ok = rp_gpu <= 10.0 and rg_gpu <= 10.0 and pv["near_tie"] and gpu["info"] == [0, 0]
    check = {"ok": bool(ok), "n": n, "bound": 10.0, "eps": "2^-23",
             "what": "factors of the last timed step vs the CPU FP64 oracle and host LAPACK",
             "potrf_scaled_residual": round(rp_gpu, 5),
             "potrf_scaled_residual_host_lapack": round(rp_cpu, 5),
             "getrf_scaled_residual": round(rg_gpu, 5),
             "getrf_scaled_residual_host_lapack": round(rg_cpu, 5),
             "pivots_vs_sgetrf": "identical" if pv["first_divergence"] is None else pv,
             "info": gpu["info"], "check_s": round(time.perf_counter() - t0, 1)}
    return base, check


def reference_arm(args):
    """--impl reference: host LAPACK spotrf + sgetrf (the reference's CPU path
    of its residual harness) at the bench's own size n, all host threads.
    Warm-up is one small pair (it only starts the BLAS threads); then as many
    of the requested steps as fit in about six minutes are timed, at least one,
    each a full POTRF + GETRF of order n."""
    thr, ver = cpu_threads()
    n = args.n
    Aw, Gw = host_inputs(2048)
    lapack_pair(Aw, Gw)
    t0 = time.perf_counter()
    lapack_pair(Aw, Gw)
    rate = (flops_potrf(2048) + flops_getrf(2048)) / (time.perf_counter() - t0)
    A, G = host_inputs(n)
    est = (flops_potrf(n) + flops_getrf(n)) / (2.0 * rate)  # larger orders run faster
    steps = max(1, min(args.steps, int(360.0 / max(est, 1e-3))))
    tot = tp_sum = tg_sum = 0.0
    for _ in range(steps):
        _, _, _, tp, tg = lapack_pair(A, G)
        tp_sum += tp
        tg_sum += tg
    tot = tp_sum + tg_sum
    value = steps * (flops_potrf(n) + flops_getrf(n)) / tot / 1e12
    return {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "steps_requested": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * tot / steps, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (same seeded input families, built on the host)",
            "impl": "reference",
            "config": {"workload": (f"host LAPACK spotrf(lower)+sgetrf at n={n} (the POTRF+GETRF "
                                    f"workload of the GPU arm), {steps} full step(s)"), "n": n},
            "potrf_tflops": round(steps * flops_potrf(n) / tp_sum / 1e12, 4),
            "getrf_tflops": round(steps * flops_getrf(n) / tg_sum / 1e12, 4),
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": thr, "kind": "port",
                             "sample": (f"SciPy OpenBLAS {ver} spotrf+sgetrf, {thr} threads, "
                                        f"n={n}, {steps} step(s) (of {args.steps} requested: "
                                        "steps beyond a six-minute budget are not run), "
                                        "warm-up one n=2048 pair")},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


# ----------------------------------------------------------------- GPU arm
class Workload:
    def __init__(self, torch, hd, n, handle, params):
        self.torch, self.hd, self.n, self.h, self.p = torch, hd, n, handle, params
        dev = "cuda"
        nn = n * n
        # SPD input: A = G G^T / n + I in FP64, rounded to FP32
        G = torch.empty(nn, dtype=torch.float32, device=dev)
        st = hd.lib().hdbf_fill_uniform(handle.ptr, G.data_ptr(), nn, 0, 0)
        assert st == 0
        T = G.view(n, n).double()  # row-major view = G^T (G is column-major)
        del G
        A64 = (T.t() @ T).div_(n)
        del T
        A64 = 0.5 * (A64 + A64.t())
        A64.diagonal().add_(1.0)
        self.spd0 = A64.float().reshape(-1).contiguous()
        del A64
        torch.cuda.empty_cache()
        self.gen0 = torch.empty(nn, dtype=torch.float32, device=dev)
        st = hd.lib().hdbf_fill_uniform(handle.ptr, self.gen0.data_ptr(), nn, 1, 0)
        assert st == 0
        self.spd = torch.empty_like(self.spd0)
        self.gen = torch.empty_like(self.gen0)
        self.ipiv = torch.zeros(n, dtype=torch.int32, device=dev)
        self.info = torch.zeros(2, dtype=torch.int32, device=dev)
        tile = params["getrf_pivot_tile"]
        self.ws_src = torch.zeros(n, dtype=torch.int32, device=dev)
        self.ws_tgt = torch.zeros(n, dtype=torch.int32, device=dev)
        self.ws_swap = torch.zeros(n * tile, dtype=torch.float32, device=dev)
        import numpy as np
        self.ws_host = [np.zeros(n, np.int32) for _ in range(4)]
        self.ws = hd.WorkspacePivot(self.ws_src.data_ptr(), self.ws_tgt.data_ptr(),
                                    self.ws_swap.data_ptr(), *[a.ctypes.data for a in self.ws_host],
                                    n, tile)
        handle.reserve(hd.lib().hdbf_workspace_bytes_for(n))
        torch.cuda.synchronize()

    def potrf(self, A):
        p, n = self.p, self.n
        self.hd.call("double_blocked_potrf_kblocked_syrk", self.h.ptr, A.data_ptr(), n, n,
                     p["potrf_nb"], p["potrf_b"], p["potrf_tk"], self.info.data_ptr())

    def getrf(self, A, ipiv):
        import ctypes
        p, n = self.p, self.n
        self.hd.call("double_blocked_getrf_batched_pivot", self.h.ptr, A.data_ptr(), n, n,
                     p["getrf_nb"], p["getrf_b"], 1, p["getrf_trsm_block"], p["getrf_mtile"],
                     ipiv.data_ptr(), self.info.data_ptr() + 4, ctypes.byref(self.ws))

    def step(self):
        self.spd.copy_(self.spd0)
        self.potrf(self.spd)
        self.gen.copy_(self.gen0)
        self.getrf(self.gen, self.ipiv)


def mixed_ir_cases(torch, hd, handle, n, cases, nrhs=16, seed=2026):
    """Time-to-solution of A x = b to FP64 backward error <= 1e-13 (configs
    of the mixed-precision workload): FP32 factors + FP64 refinement versus
    tensor-core (BF16/FP16) factors + FP64 refinement, SPD and general A with
    singular values log-spaced in [1, kappa] (Q from QR of an N(0,1) matrix)."""
    import ctypes
    gen = torch.Generator(device="cuda")
    out = {}
    mats = {}

    def matrix(kind, kappa):
        key = (kind, kappa)
        if key in mats:
            return mats[key]
        mats.clear()
        torch.cuda.empty_cache()
        gen.manual_seed(seed)
        Q, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=gen))
        lam = torch.logspace(0.0, float(np.log10(kappa)), n, dtype=torch.float64, device="cuda")
        if kind == "spd":
            A = (Q * lam) @ Q.t()
            A = 0.5 * (A + A.t())
        else:
            V, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=gen))
            A = (Q * lam) @ V.t()
        del Q
        A = A.t().contiguous()  # column-major storage
        B = torch.randn(nrhs, n, dtype=torch.float64, device="cuda", generator=gen).contiguous()
        mats[key] = (A, B)
        return A, B

    def independent_berr(A, B, X):
        """max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf)
        recomputed with torch's FP64 GEMM on the device, independent of the
        library's refinement kernels (A, B, X column-major storage)."""
        Am = A.view(n, n).t()
        Bm, Xm = B.view(nrhs, n).t(), X.view(nrhs, n).t()
        R = Bm - Am @ Xm
        an = float(Am.abs().sum(dim=1).max())
        num = R.abs().amax(dim=0)
        den = an * Xm.abs().amax(dim=0) + Bm.abs().amax(dim=0)
        return float((num / den).max())

    def run(kind, A, B, X, prec, method):
        if method == "gmres":
            fn = "hdbf_dposv_mixed_gmres" if kind == "spd" else "hdbf_dgesv_mixed_gmres"
        elif method == "auto":
            fn = "hdbf_dposv_mixed_auto" if kind == "spd" else "hdbf_dgesv_mixed_auto"
        else:
            fn = "hdbf_dposv_mixed" if kind == "spd" else "hdbf_dgesv_mixed"
        info = hd.IrInfo()
        if method == "gmres":
            args = (handle.ptr, hd.PREC[prec], A.data_ptr(), n, n, nrhs, B.data_ptr(), n,
                    X.data_ptr(), n, ctypes.c_double(1e-13), 10, 30, ctypes.c_double(1e-4),
                    ctypes.byref(info))
        elif method == "auto":
            args = (handle.ptr, hd.PREC[prec], A.data_ptr(), n, n, nrhs, B.data_ptr(), n,
                    X.data_ptr(), n, ctypes.c_double(1e-13), 30, ctypes.byref(info))
        else:
            args = (handle.ptr, hd.PREC[prec], 1, A.data_ptr(), n, n, nrhs, B.data_ptr(), n,
                    X.data_ptr(), n, ctypes.c_double(1e-13), 30, ctypes.byref(info))
        hd.call(fn, *args)  # builds the graphs and the workspace
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = hd.call(fn, *args)
        e1.record()
        torch.cuda.synchronize()
        return {"method": method, "precision": prec, "ms": round(e0.elapsed_time(e1), 2),
                "backward_error_independent": independent_berr(A, B, X),
                "fallback_panels": int(info.fallback_panels),
                "status": int(st), "converged": int(info.converged),
                "iterations": int(info.iterations), "inner_iterations": int(info.inner_iterations),
                "backward_error": float(info.backward_error),
                "final_precision": int(info.final_precision),
                "factorizations": int(info.factorizations),
                "factor_ms": round(info.factor_ms, 2), "refine_ms": round(info.refine_ms, 2),
                "history": [float(f"{info.history[i]:.3e}")
                            for i in range(min(64, int(info.iterations) + 1))]}

    fp32_done = {}
    for kind, kappa, prec, method in cases:
        A, B = matrix(kind, kappa)
        X = torch.zeros(nrhs, n, dtype=torch.float64, device="cuda")
        if (kind, kappa) not in fp32_done:
            # FP32 reference: the faster converged of classical IR and GMRES-IR
            cand = [run(kind, A, B, X, "fp32", mth) for mth in ("ir", "gmres")]
            ok = [c for c in cand if c["converged"] and c["backward_error"] <= 1e-13
                  and c["backward_error_independent"] <= 1e-13]
            fp32_done[(kind, kappa)] = (min(ok, key=lambda c: c["ms"]) if ok else
                                        min(cand, key=lambda c: c["ms"]), cand)
        r32, alts = fp32_done[(kind, kappa)]
        # "auto": the library's adaptive refinement (classical IR, then
        # GMRES-IR, then a higher factorization precision), one call
        rm = run(kind, A, B, X, prec, method)
        flops = (n ** 3 / 3.0) if kind == "spd" else (2.0 * n ** 3 / 3.0)
        key = f"{'potrf' if kind == 'spd' else 'getrf'}_k{kappa:.0e}_{prec}_{method}"
        out[key] = {
            "fp32_ir": r32, "fp32_alternatives": alts, "mixed_ir": rm,
            "speedup_time_to_solution": round(r32["ms"] / rm["ms"], 3) if rm["ms"] > 0 else None,
            "mixed_effective_tflops": round(flops / (rm["ms"] / 1e3) / 1e12, 2),
            "fp32_effective_tflops": round(flops / (r32["ms"] / 1e3) / 1e12, 2)}
    mats.clear()
    torch.cuda.empty_cache()
    return out


def config2(args):
    """Mixed precision + FP64 refinement over the whole config-2 grid (opt-in,
    ``--config2``): n in {16384, 32768}, SPD and general A with singular
    values log-spaced in [1, kappa], kappa in {1e2, 1e4, 1e6}, BF16 and FP16
    trailing updates, nrhs = 16.  Each cell: the FP32 reference (faster
    converged of classical IR and GMRES-IR), then one call of the library's
    adaptive refinement from the mixed factorization (classical IR, GMRES-IR
    from the first stalled step, a higher factorization precision when GMRES
    stalls; hdbf_d{po,ge}sv_mixed_auto) to 1e-13; refinement iterations,
    final precision, the library's and an independently recomputed FP64
    backward error, and the time-to-solution speed-up.  One JSON line per
    order, then a summary."""
    import torch
    import hygondoubleblockedfactorizations_b200 as hd
    torch.cuda.set_device(0)
    handle = hd.Handle(torch.cuda.current_stream().cuda_stream)
    summary = []
    for n in [int(x) for x in args.config2_sizes.split(",")]:
        cases = [(kind, kappa, prec, "auto") for kind in ("spd", "gen")
                 for kappa in (1e2, 1e4, 1e6) for prec in ("bf16", "fp16")]
        res = mixed_ir_cases(torch, hd, handle, n, cases)
        print(json.dumps({"config2_n": n, "cells": res}), flush=True)
        for key, v in res.items():
            m = v["mixed_ir"]
            summary.append({"n": n, "cell": key, "method": m["method"],
                            "final_precision": m["final_precision"],
                            "factorizations": m["factorizations"],
                            "iterations": m["iterations"],
                            "inner_iterations": m["inner_iterations"],
                            "backward_error": m["backward_error"],
                            "backward_error_independent": m["backward_error_independent"],
                            "converged": bool(m["converged"] and m["backward_error"] <= 1e-13
                                              and m["backward_error_independent"] <= 1e-13),
                            "fallback_panels": m["fallback_panels"],
                            "speedup_time_to_solution": v["speedup_time_to_solution"],
                            "fp32_ms": v["fp32_ir"]["ms"], "mixed_ms": m["ms"]})
    handle.close()
    print(json.dumps({"config2": summary}), flush=True)


def fp64_case(torch, hd, handle, n=8192, reps=2):
    """FP64 twins at n=8192: double_blocked_potrf_double (nb 2048, b 256) and
    double_blocked_getrf_double_batched_pivot (nb 2048, b 256, iterative outer
    TRSM) on the bench's input families drawn in FP32 by the seeded generator
    and widened to FP64 (SPD G G^T/n + I, general U[-1,1)).  Device time per
    call with CUDA events (mean of `reps` after one warm-up, the input restored
    from a pristine copy outside the timed region); TFLOP/s with n^3/3 and
    2n^3/3 against the nominal FP64 FMA peak; FP64 residuals
    ||A - LL^T||_F / (||A||_F n eps64) and ||PA - LU||_F / (||A||_F n eps64)."""
    import ctypes

    import numpy as np
    P = ctypes.c_void_p
    dev = torch.device("cuda")

    def draw(seed):
        x = torch.empty(n * n, dtype=torch.float32, device=dev)
        hd.lib().hdbf_fill_uniform(handle.ptr, P(x.data_ptr()), n * n, seed, 0)
        return x.view(n, n).t().double()  # column-major storage: element (r, c) at c*n + r

    G = draw(0)
    spd0 = (G @ G.t()) / n + torch.eye(n, dtype=torch.float64, device=dev)
    spd0 = 0.5 * (spd0 + spd0.t())
    gen0 = draw(1)
    del G
    # the library reads column-major: keep each matrix as the transpose's storage
    spd_cm = spd0.t().contiguous()
    gen_cm = gen0.t().contiguous()
    A = torch.empty_like(spd_cm)
    info = torch.zeros(2, dtype=torch.int32, device=dev)
    ipiv = torch.zeros(n, dtype=torch.int32, device=dev)
    tile = 16
    keep = [torch.zeros(n, dtype=torch.int32, device=dev),
            torch.zeros(n, dtype=torch.int32, device=dev),
            torch.zeros(n * tile, dtype=torch.float64, device=dev)]
    host = [np.zeros(n, np.int32) for _ in range(4)]
    ws = hd.WorkspacePivot(keep[0].data_ptr(), keep[1].data_ptr(), keep[2].data_ptr(),
                           *[h.ctypes.data for h in host], n, tile)

    def potrf():
        hd.call("double_blocked_potrf_double", handle.ptr, P(A.data_ptr()), n, n, 2048, 256,
                P(info.data_ptr()))

    def getrf():
        hd.call("double_blocked_getrf_double_batched_pivot", handle.ptr, P(A.data_ptr()), n, n,
                2048, 256, 1, 0, 0, P(ipiv.data_ptr()), P(info.data_ptr() + 4), ctypes.byref(ws))

    def timed(src, fn):
        times = []
        for r in range(reps + 1):
            A.copy_(src)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            if r > 0:
                times.append(e0.elapsed_time(e1))
        handle.check()
        return sum(times) / len(times)

    eps = 2.0 ** -52
    ms_p = timed(spd_cm, potrf)
    L = torch.tril(A.t())
    res_p = float(torch.linalg.norm(spd0 - L @ L.t()) / torch.linalg.norm(spd0)) / (n * eps)
    del L
    ms_g = timed(gen_cm, getrf)
    LU = A.t()
    Lm = torch.tril(LU, -1) + torch.eye(n, dtype=torch.float64, device=dev)
    Um = torch.triu(LU)
    perm = np.arange(n)
    piv = ipiv.cpu().numpy()
    for i in range(n):
        p = int(piv[i]) - 1
        perm[i], perm[p] = perm[p], perm[i]
    PA = gen0[torch.from_numpy(perm).to(dev)]
    res_g = float(torch.linalg.norm(PA - Lm @ Um) / torch.linalg.norm(gen0)) / (n * eps)
    infos = info.cpu().tolist()
    props = torch.cuda.get_device_properties(0)
    peak = props.multi_processor_count * 64 * 2 * 1965e6 / 1e12
    tp = n ** 3 / 3.0 / (ms_p / 1e3) / 1e12
    tg = 2.0 * n ** 3 / 3.0 / (ms_g / 1e3) / 1e12
    return {"workload": f"n={n} double_blocked_potrf_double(nb 2048, b 256) + "
                        "double_blocked_getrf_double_batched_pivot(nb 2048, b 256, iterative "
                        "outer TRSM)",
            "potrf_ms": round(ms_p, 3), "getrf_ms": round(ms_g, 3),
            "potrf_tflops": round(tp, 3), "getrf_tflops": round(tg, 3),
            "peak_tflops": round(peak, 2),
            "peak_source": f"nominal: {props.multi_processor_count} SMs x 64 FP64 FMA/clk x 2 "
                           "x 1965 MHz (no measured FP64 peak on this pool)",
            "frac_potrf": round(tp / peak, 4), "frac_getrf": round(tg / peak, 4),
            "scaled_residual": {"potrf": round(res_p, 4), "getrf": round(res_g, 4)},
            "info": infos, "eps": "2^-52"}


def batched_case(torch, hd, handle, reps=5):
    """The uneven batch in one persistent launch: 4096 SPD systems with
    n ~ U[16, 512] and 2048 general systems with n ~ U[32, 768] (seed 3), one
    N(0,1) right-hand side each; CTA size picked by the autotuner.  Checks
    every system on the GPU in FP64: scaled factorization residual
    ||A - LL^T||_F / (||A||_F n eps) or ||PA - LU||_F / (||A||_F n eps), and the
    normwise backward error of the solution."""
    from hygondoubleblockedfactorizations_b200 import batch as bm
    from hygondoubleblockedfactorizations_b200 import tuner
    ops, ns = bm.config3_sizes()
    b = bm.DeviceBatch(torch, ops, ns)
    bm.fill_batch(torch, handle, b, 3)
    best, tuned = tuner.tune_batched(torch, handle, b, reps=2)
    times = []
    for _ in range(reps):
        bm.restore(b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = b.run(handle, best)
        e1.record()
        torch.cuda.synchronize()
        assert st == 0
        times.append(e0.elapsed_time(e1))
    ms = sorted(times)[len(times) // 2]
    info = b.info.cpu().numpy()
    piv = b.ipiv_buf.cpu().numpy()
    eps = 2.0 ** -23
    worst = {"potrf": 0.0, "getrf": 0.0}
    worst_be = 0.0
    for i in range(b.count):
        n = int(b.ns[i])
        o = int(b.offsets[i])
        A0 = b.A0[o:o + n * n].view(n, n).t().double()
        F = b.A[o:o + n * n].view(n, n).t().double()
        r0 = int(b.roffsets[i])
        x = b.b[r0:r0 + n].double()
        rhs = b.b0[r0:r0 + n].double()
        if b.ops[i] == 0:
            L = torch.tril(F)
            res = torch.linalg.matrix_norm(A0 - L @ L.t()) / torch.linalg.matrix_norm(A0)
            key = "potrf"
        else:
            L = torch.tril(F, -1) + torch.eye(n, dtype=torch.float64, device="cuda")
            U = torch.triu(F)
            perm = np.arange(n)
            for j, p in enumerate(piv[r0:r0 + n] - 1):
                perm[j], perm[p] = perm[p], perm[j]
            PA = A0[torch.from_numpy(perm).cuda()]
            res = torch.linalg.matrix_norm(PA - L @ U) / torch.linalg.matrix_norm(A0)
            key = "getrf"
        worst[key] = max(worst[key], float(res) / (n * eps))
        r = rhs - A0 @ x
        an = float(A0.abs().sum(1).max())
        be = float(r.abs().max()) / (an * float(x.abs().max()) + float(rhs.abs().max()))
        worst_be = max(worst_be, be)
    flops = b.flops()
    return {"workload": "4096 SPD n~U[16,512] + 2048 general n~U[32,768], 1 RHS each, one launch",
            "variant": int(best), "variant_ms": {str(k): round(v, 3) for k, v in tuned.items()},
            "ms": round(ms, 3), "tflops": round(flops / (ms / 1e3) / 1e12, 3),
            "gflop": round(flops / 1e9, 2), "info_nonzero": int((info != 0).sum()),
            "worst_scaled_residual": {k: round(v, 4) for k, v in worst.items()},
            "worst_backward_error": worst_be, "eps": "2^-23"}


# The reference's published K100 AI times (ms) of the same two algorithms
# (POTRF DoubleBlock+KBSYRK, GETRF DB-LU+BatchedPivot+MGEMM), per order.
REF_PUBLISHED_SWEEP_MS = {8192: {"potrf": 32.5}, 16384: {"potrf": 108.9, "getrf": 492.6},
                          32768: {"potrf": 565.6, "getrf": 2152.1},
                          49152: {"potrf": 1655.2, "getrf": 6651.2}}


def sweep(args):
    """Config-1 sweep (opt-in, ``--sweep``): POTRF on G G^T/n + I and pivoted
    GETRF on U[-1,1) for each order, with the bench's blocks (clamped to n).
    Per order: device time of each factorization (mean of ``--steps`` after
    ``--warmup``), then the checker on the host -- host LAPACK spotrf/sgetrf on
    the same FP32 inputs (timed: the CPU baseline at that order), CPU FP64
    scaled residuals of both factorizations (<= 10), GPU pivots vs sgetrf's
    (identical, or a first divergence at an FP32 near-tie).  One JSON line per
    order, then a summary line; exits non-zero if any order fails."""
    import torch
    import hygondoubleblockedfactorizations_b200 as hd
    import oracle  # checker and CPU baseline leg only
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    thr, ver = cpu_threads()
    rows = []
    for n in [int(x) for x in args.sweep_sizes.split(",")]:
        handle = hd.Handle(stream.cuda_stream)
        wl = Workload(torch, hd, n, handle, dict(DEFAULTS))
        times = {}
        for op in ("potrf", "getrf"):
            src, dst = (wl.spd0, wl.spd) if op == "potrf" else (wl.gen0, wl.gen)
            run = (lambda: wl.potrf(dst)) if op == "potrf" else (lambda: wl.getrf(dst, wl.ipiv))
            ts = []
            for r in range(args.warmup + args.steps):
                dst.copy_(src)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                run()
                e1.record(stream)
                torch.cuda.synchronize()
                if r >= args.warmup:
                    ts.append(e0.elapsed_time(e1))
            times[op] = sum(ts) / len(ts)
        handle.check("sweep")
        info = wl.info.cpu().tolist()
        dev_err = handle.device_errors()
        from scipy.linalg import lapack
        row = {"n": n, "info": info, "device_errors": dev_err, "blocks": {
            "potrf": [min(n, DEFAULTS["potrf_nb"]), DEFAULTS["potrf_b"]],
            "getrf": [min(n, DEFAULTS["getrf_nb"]), DEFAULTS["getrf_b"]]}}
        # POTRF: host copies, LAPACK, residuals (one matrix family at a time)
        A = wl.spd0.cpu().numpy().reshape(n, n).T
        L = wl.spd.cpu().numpy().reshape(n, n).T
        t0 = time.perf_counter()
        Lh, inf_h = lapack.spotrf(A, lower=1, clean=0, overwrite_a=0)
        tp = time.perf_counter() - t0
        rp = oracle.scaled(oracle.potrf_residual_tiled(L, A), n)
        rph = oracle.scaled(oracle.potrf_residual_tiled(Lh, A), n)
        del A, L, Lh
        G = wl.gen0.cpu().numpy().reshape(n, n).T
        LU = wl.gen.cpu().numpy().reshape(n, n).T
        ipiv = wl.ipiv.cpu().numpy().copy()
        del wl
        handle.close()
        torch.cuda.empty_cache()
        t0 = time.perf_counter()
        LUh, pivh, inf_g = lapack.sgetrf(G, overwrite_a=0)
        tg = time.perf_counter() - t0
        pivh = (pivh + 1).astype(np.int32)
        rg = oracle.scaled(oracle.getrf_residual_tiled(LU, G, ipiv), n)
        rgh = oracle.scaled(oracle.getrf_residual_tiled(LUh, G, pivh), n)
        del LU, LUh
        pv = oracle.pivot_agreement(G, pivh, ipiv)
        del G
        ok = info == [0, 0] and dev_err == 0 and rp <= 10.0 and rg <= 10.0 and pv["near_tie"]
        pub = REF_PUBLISHED_SWEEP_MS.get(n, {})
        row.update({
            "ok": bool(ok),
            "potrf_ms": round(times["potrf"], 3),
            "potrf_tflops": round(flops_potrf(n) / (times["potrf"] / 1e3) / 1e12, 3),
            "getrf_ms": round(times["getrf"], 3),
            "getrf_tflops": round(flops_getrf(n) / (times["getrf"] / 1e3) / 1e12, 3),
            "potrf_scaled_residual": round(rp, 5), "potrf_scaled_residual_host_lapack": round(rph, 5),
            "getrf_scaled_residual": round(rg, 5), "getrf_scaled_residual_host_lapack": round(rgh, 5),
            "pivots_vs_sgetrf": "identical" if pv["first_divergence"] is None else pv,
            "cpu_baseline": {"potrf_ms": round(1e3 * tp, 1), "getrf_ms": round(1e3 * tg, 1),
                             "potrf_tflops": round(flops_potrf(n) / tp / 1e12, 4),
                             "getrf_tflops": round(flops_getrf(n) / tg / 1e12, 4),
                             "cores": thr, "kind": "port",
                             "sample": f"SciPy OpenBLAS {ver} spotrf+sgetrf, {thr} threads, 1 run"},
            "reference_published_k100_ms": pub or None})
        rows.append(row)
        print(json.dumps(row), flush=True)
    bad = [r["n"] for r in rows if not r["ok"]]
    print(json.dumps({"sweep": "config-1 FP32 POTRF + GETRF", "orders": [r["n"] for r in rows],
                      "all_ok": not bad, "failed": bad, "steps": args.steps,
                      "warmup": args.warmup, "eps": "2^-23", "bound": 10.0}), flush=True)
    if bad:
        raise SystemExit(f"sweep check failed at n={bad}")


def gpu_index():
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    if vis and vis.split(",")[0].strip().isdigit():
        lr = int(os.environ.get("LOCAL_RANK", "0"))
        ids = [v.strip() for v in vis.split(",")]
        return int(ids[0]) if len(ids) == 1 else int(ids[lr])
    return int(os.environ.get("LOCAL_RANK", "0"))


# Blocks: the fastest FP32 candidates of the exhaustive B200 sweep at n = 32768
# (tests/golden/selector_records_b200.json; the learned selector picks the same).
DEFAULTS = dict(potrf_nb=4096, potrf_b=512, potrf_tk=0, getrf_nb=8192, getrf_b=1024,
                getrf_trsm_block=0, getrf_mtile=0, getrf_pivot_tile=64)

# The reference's published K100 AI numbers at n = 32768 (its paper-final scaling runs):
# POTRF DoubleBlock+KBSYRK 565.6 ms, GETRF DB-LU+BatchedPivot+MGEMM 2152.1 ms.
REF_PUBLISHED_MS = {"potrf": 565.6, "getrf": 2152.1}


def run_ours(args, rank, world):
    import torch
    import hygondoubleblockedfactorizations_b200 as hd
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    stream = torch.cuda.current_stream()
    handle = hd.Handle(stream.cuda_stream)
    n = args.n
    params = dict(DEFAULTS)
    wl = Workload(torch, hd, n, handle, params)
    dist = world > 1
    if dist:
        import torch.distributed as tdist

    def barrier():
        if dist:
            tdist.barrier()
        torch.cuda.synchronize()

    # warm-up (also checks the factorizations succeeded).  The library records
    # each factorization as a CUDA graph on first use; warming up with the
    # event profiler on builds the profiled graphs used in the timed region.
    handle.profile_begin()
    for _ in range(args.warmup):
        wl.step()
    torch.cuda.synchronize()
    handle.profile_end()
    info = wl.info.cpu().tolist()
    handle.check("warm-up")
    if info != [0, 0] or handle.device_errors() != 0:
        raise SystemExit(f"factorization failed during warm-up: info={info}")

    # ---- timed region (device-resident inputs)
    sampler = ClockSampler(gpu_index()) if rank == 0 else None
    barrier()
    if sampler:
        sampler.start()
        time.sleep(0.3)
    launches0 = handle.launches()
    handle.profile_begin()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        wl.step()
    ev1.record(stream)
    torch.cuda.synchronize()
    prof = handle.profile_end()
    launches = handle.launches() - launches0
    clocks = sampler.stop() if sampler else None
    barrier()
    ms = ev0.elapsed_time(ev1)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    ms_max = float(t.item())
    info = wl.info.cpu().tolist()
    # the last timed step's factors, kept for the check against the oracle
    # (later legs reuse the device buffers)
    factors = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        factors = {"L": wl.spd.cpu().numpy().reshape(n, n).T,
                   "LU": wl.gen.cpu().numpy().reshape(n, n).T,
                   "ipiv": wl.ipiv.cpu().numpy().copy(), "info": info,
                   "A": wl.spd0.cpu().numpy().reshape(n, n).T,
                   "G": wl.gen0.cpu().numpy().reshape(n, n).T}

    # per-op split (one extra untimed step, events between the two ops)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record(stream); wl.spd.copy_(wl.spd0); wl.potrf(wl.spd); e[1].record(stream)
    e[2].record(stream); wl.gen.copy_(wl.gen0); wl.getrf(wl.gen, wl.ipiv); e[3].record(stream)
    torch.cuda.synchronize()
    ms_potrf, ms_getrf = e[0].elapsed_time(e[1]), e[2].elapsed_time(e[3])

    # ---- e2e: pinned host buffers through the C ABI
    e2e = None
    if not args.skip_e2e:
        nn = n * n
        h_spd = torch.empty(nn, dtype=torch.float32, pin_memory=True)
        h_gen = torch.empty(nn, dtype=torch.float32, pin_memory=True)
        h_spd.copy_(wl.spd0.cpu())
        h_gen.copy_(wl.gen0.cpu())
        o_spd = torch.empty(nn, dtype=torch.float32, pin_memory=True)
        o_gen = torch.empty(nn, dtype=torch.float32, pin_memory=True)
        o_piv = torch.empty(n, dtype=torch.int32, pin_memory=True)
        o_info = torch.empty(2, dtype=torch.int32, pin_memory=True)

        # Copies run on a second stream so they overlap the other matrix's
        # factorization: GETRF's input uploads during POTRF, POTRF's factor
        # downloads during GETRF.  Every copy stays inside the timed region
        # (the compute stream joins the copy stream before the end event).
        cstream = torch.cuda.Stream()
        ev = [torch.cuda.Event() for _ in range(4)]

        def e2e_step():
            with torch.cuda.stream(cstream):
                cstream.wait_stream(stream)          # previous step's users of the buffers
                wl.spd.copy_(h_spd, non_blocking=True)
                ev[0].record(cstream)
                wl.gen.copy_(h_gen, non_blocking=True)
                ev[1].record(cstream)
            stream.wait_event(ev[0])
            wl.potrf(wl.spd)
            ev[2].record(stream)
            stream.wait_event(ev[1])
            wl.getrf(wl.gen, wl.ipiv)
            ev[3].record(stream)
            with torch.cuda.stream(cstream):
                cstream.wait_event(ev[2])
                o_spd.copy_(wl.spd, non_blocking=True)
                cstream.wait_event(ev[3])
                o_gen.copy_(wl.gen, non_blocking=True)
                o_piv.copy_(wl.ipiv, non_blocking=True)
                o_info.copy_(wl.info, non_blocking=True)
            stream.wait_stream(cstream)

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        ev1.record(stream)
        torch.cuda.synchronize()
        t2 = torch.tensor([ev0.elapsed_time(ev1)], dtype=torch.float64, device="cuda")
        if dist:
            tdist.all_reduce(t2, op=tdist.ReduceOp.MAX)
        e2e_ms = float(t2.item())
        assert o_info.tolist() == [0, 0]
        e2e = {"value": round(world * args.steps * (flops_potrf(n) + flops_getrf(n)) / (e2e_ms / 1e3) / 1e12, 4),
               "unit": UNIT, "h2d_bytes_per_step": 2 * nn * 4,
               "d2h_bytes_per_step": 2 * nn * 4 + n * 4 + 8,
               "ms_per_step": round(e2e_ms / args.steps, 3)}
        del h_spd, h_gen, o_spd, o_gen

    mixed = None
    if not args.skip_mixed and world == 1:
        cases = [("spd", 1e2, "bf16", "ir"), ("spd", 1e2, "fp16", "ir"),
                 ("gen", 1e2, "fp16", "gmres"), ("gen", 1e2, "bf16", "auto"),
                 ("gen", 1e2, "fp16x3", "ir"), ("gen", 1e4, "fp16", "auto"),
                 ("spd", 1e6, "fp16x3", "ir"), ("gen", 1e6, "fp16x3", "gmres")]
        mixed = mixed_ir_cases(torch, hd, handle, n, cases)
        best = {}
        for key, v in mixed.items():
            op = key.split("_")[0]
            m = v["mixed_ir"]
            if (m["converged"] and m["backward_error"] <= 1e-13
                    and m["backward_error_independent"] <= 1e-13):
                if op not in best or v["speedup_time_to_solution"] > best[op]["speedup"]:
                    best[op] = {"case": key, "speedup": v["speedup_time_to_solution"]}
        mixed["best_speedup_at_1e-13"] = best
        # tensor-core roofline: one profiled BF16 mixed POTRF of the bench's SPD matrix
        import ctypes
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        tc_peak = peaks.get("bf16_tflops", 1590.0)
        wl.spd.copy_(wl.spd0)
        hd.lib().hdbf_spotrf_mixed(handle.ptr, hd.PREC["bf16"], ctypes.c_void_p(wl.spd.data_ptr()),
                                   n, n, 1024, ctypes.c_void_p(wl.info.data_ptr()))
        wl.spd.copy_(wl.spd0)
        torch.cuda.synchronize()
        handle.profile_begin()
        hd.lib().hdbf_spotrf_mixed(handle.ptr, hd.PREC["bf16"], ctypes.c_void_p(wl.spd.data_ptr()),
                                   n, n, 1024, ctypes.c_void_p(wl.info.data_ptr()))
        tprof = handle.profile_end()
        tc = tprof.get("tc_gemm_kernels")
        tc_name = ("tc_gemm_sub_kernel" if os.environ.get("HDBF_TC_KERNEL", "0").strip() not in ("", "0")
                   else "tc_gemm_persistent_kernel")
        if tc:
            nl, tms, fl, by = tc
            ach = fl / (tms / 1e3) / 1e12
            mixed["tensor_roofline"] = {
                "bound": "tensor", "kernel": tc_name, "workload":
                f"BF16 mixed POTRF n={n} panel 1024 (all tcgen05 updates: narrow in-pair "
                "updates and K=2048 trailing SYRK updates)",
                "achieved": round(ach, 1), "peak": tc_peak, "unit": "TFLOP/s",
                "frac": round(ach / tc_peak, 4), "launches": nl,
                "avg_launch_ms": round(tms / nl, 4),
                "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else "fallback"}

    batched = None
    if not args.skip_batched and world == 1:
        batched = batched_case(torch, hd, handle)

    fp64 = None
    if not args.skip_fp64 and world == 1:
        try:
            fp64 = fp64_case(torch, hd, handle)
        except Exception as exc:  # reported in the line, never hides the FP32 result
            fp64 = {"error": f"{type(exc).__name__}: {exc}"}

    total_flops = world * args.steps * (flops_potrf(n) + flops_getrf(n))
    value = total_flops / (ms_max / 1e3) / 1e12
    vs_baseline = None
    if n == 32768:
        ref_rate = (flops_potrf(n) + flops_getrf(n)) / (
            (REF_PUBLISHED_MS["potrf"] + REF_PUBLISHED_MS["getrf"]) / 1e3) / 1e12
        vs_baseline = round(value / (world * ref_rate), 4)

    # roofline of the dominant kernel
    dom = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    props = torch.cuda.get_device_properties(0)
    sms = props.multi_processor_count
    max_mhz = (clocks or {}).get("sm_max_mhz") or 1965.0
    peak = sms * 128 * 2 * max_mhz * 1e6 / 1e12
    roof = None
    if dom:
        name, (nl, tms, fl, by) = dom
        achieved = fl / (tms / 1e3) / 1e12
        # DRAM bytes per algorithmic flop of sgemm_sub_kernel, measured by ncu
        # (dram__bytes_read.sum + dram__bytes_write.sum) on the largest launch
        # of a POTRF n=16384: 852.5 MB over 2.75e11 flop (FMA-pipe count).
        bytes_per_flop = 852.5e6 / 2.75e11
        roof = {"bound": "fp32_simt", "kernel": name, "achieved": round(achieved, 3),
                "peak": round(peak, 2), "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                "traffic": round(fl / nl * bytes_per_flop) if name == "sgemm_sub_kernel" else None,
                "traffic_unit": "bytes per average launch (ncu bytes/flop of a captured "
                                "n=16384 launch x this launch's algorithmic flops)",
                "algorithmic_flops_per_launch": round(fl / nl),
                "launches": nl, "avg_launch_ms": round(tms / nl, 4),
                "share_of_device_time": round(tms / sum(v[1] for v in prof.values()), 4),
                "peak_source": (f"{sms} SMs x 128 FP32 lanes x 2 flop x {max_mhz:.0f} MHz max SM "
                                "clock (measured-peaks file has no FP32 SIMT figure)")}
        if clocks and clocks.get("sm_mhz"):
            roof["frac_at_median_clock"] = round(achieved / (peak * clocks["sm_mhz"] / max_mhz), 4)
    kernels = {k: {"launches": v[0], "ms": round(v[1], 3),
                   "tflops": round(v[2] / (v[1] / 1e3) / 1e12, 3) if v[1] > 0 and v[2] > 0 else None,
                   "gbs": round(v[3] / (v[1] / 1e3) / 1e9, 1) if v[1] > 0 and v[3] > 0 else None}
               for k, v in prof.items()}

    out = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": vs_baseline,
           "vs_baseline_ref": ("reference's published K100 AI POTRF 565.6 ms + GETRF 2152.1 ms "
                               "at n=32768 = 12.95 TFLOP/s (other hardware)"),
           "dtype": "f32",
           "data": "synthetic (seeded counter-based generator; SPD G G^T/n+I seed 0, general U[-1,1) seed 1)",
           "config": {"workload": f"n={n} POTRF(double_blocked_potrf_kblocked_syrk nb={params['potrf_nb']} b={params['potrf_b']}) + GETRF(double_blocked_getrf_batched_pivot nb={params['getrf_nb']} b={params['getrf_b']}, iterative outer TRSM)",
                      "n": n, "lda": n, "l2_flush": "inputs (2 x 4.3 GB) exceed L2; restored from pristine copies each step",
                      "parallelism": f"replicas x{world}", **params},
           "potrf_ms": round(ms_potrf, 3), "getrf_ms": round(ms_getrf, 3),
           "potrf_tflops": round(flops_potrf(n) / (ms_potrf / 1e3) / 1e12, 3),
           "getrf_tflops": round(flops_getrf(n) / (ms_getrf / 1e3) / 1e12, 3),
           "info": info, "gpu_launches": launches, "kernels": kernels,
           "roofline": roof, "clocks": clocks, "e2e": e2e, "mixed_ir": mixed,
           "batched": batched, "fp64": fp64}
    return out, handle, factors


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", type=int, default=32768)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-mixed", action="store_true")
    ap.add_argument("--skip-batched", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--sweep", action="store_true",
                    help="config-1 sweep with oracle checks instead of the bench line")
    ap.add_argument("--sweep-sizes", default="4096,8192,16384,32768,49152")
    ap.add_argument("--config2", action="store_true",
                    help="mixed precision + IR over the whole config-2 grid")
    ap.add_argument("--config2-sizes", default="16384,32768")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(reference_arm(args)), flush=True)
        return

    if args.sweep:
        sweep(args)
        return
    if args.config2:
        config2(args)
        return

    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    out, handle, factors = run_ours(args, rank, world)
    parity_ok = True
    if factors is not None:
        handle.close()
        handle = None
        base, check = cpu_baseline_and_check(args.n, factors.pop("A"), factors.pop("G"), factors)
        out["cpu_baseline"] = base
        out["parity"] = check
        parity_ok = check["ok"]
    if rank == 0:
        print(json.dumps(out), flush=True)
    if handle is not None:
        handle.close()
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()
    if not parity_ok:
        raise SystemExit("parity check of the timed factors failed (see the line's parity object)")


if __name__ == "__main__":
    main()
