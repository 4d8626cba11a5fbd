"""Regenerate the golden fixtures in this directory.

    python tests/golden/make_golden.py

residual_ref.json  -- CPU FP64 residuals computed by the REFERENCE's own header
                      (include/utils/benchmark/cpu_fp64_residual.h, compiled in
                      place into oracle/_ref by `make -C oracle ref`) on seeded
                      factor/original pairs; inputs are regenerated from the
                      seeds by gen_case() below.
lapack_f32.npz     -- host LAPACK (SciPy OpenBLAS) sgetrf pivots / info and
                      scaled residuals of sgetrf and spotrf on the seeded input
                      families (general U[-1,1) seed 1, SPD G G^T/n + I seed 0).
Needs the reference checkout ($HDBF_REFERENCE_ROOT, else /root/reference) only
for residual_ref.json.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

RES_CASES = []
for n in (1, 2, 3, 5, 11, 37, 64, 129):
    for pad in (0, 3):
        for kind in ("potrf", "getrf_piv", "getrf_nopiv"):
            for dt in ("f32", "f64"):
                for tile in (1, 3, 512):
                    if n > 40 and tile == 1:
                        continue
                    RES_CASES.append(dict(n=n, lda=n + pad, kind=kind, dtype=dt, tile=tile,
                                          seed=1000 + len(RES_CASES)))


def gen_case(c):
    """Seeded factor/original/pivots for one residual case (flat, lda-strided)."""
    n, lda = c["n"], c["lda"]
    dt = np.float32 if c["dtype"] == "f32" else np.float64
    rng = np.random.default_rng(c["seed"])
    F = rng.uniform(-1, 1, size=(lda, n)).astype(dt)
    A = rng.uniform(-1, 1, size=(lda, n)).astype(dt)
    F[n:, :] = np.nan  # padding must never be read
    A[n:, :] = np.nan
    piv = None
    if c["kind"] == "getrf_piv":
        piv = np.array([rng.integers(r + 1, n + 1) for r in range(n)], dtype=np.int32)
    return F.ravel(order="F"), A.ravel(order="F"), piv


def residual(c, impl):
    F, A, piv = gen_case(c)
    if c["kind"] == "potrf":
        return oracle.potrf_residual(F, A, c["n"], c["lda"], tile=c["tile"], impl=impl)
    return oracle.getrf_residual(F, A, piv, c["n"], c["lda"], pivoting=c["kind"] == "getrf_piv",
                                 tile=c["tile"], impl=impl)


LAPACK_N = (64, 256, 512, 1024, 2048)


def main():
    if oracle.ref_lib() is None:
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    out = []
    for c in RES_CASES:
        out.append(dict(c, value=residual(c, "ref")))
    with open(os.path.join(HERE, "residual_ref.json"), "w") as f:
        json.dump(out, f, indent=0)
    arrays = {}
    for n in LAPACK_N:
        G = oracle.general_uniform(n, 1)
        lu, ipiv, info = oracle.lapack_sgetrf(G)
        arrays[f"getrf_ipiv_{n}"] = ipiv
        arrays[f"getrf_info_{n}"] = np.int32(info)
        arrays[f"getrf_scaled_{n}"] = np.float64(oracle.scaled(oracle.getrf_residual_blas(lu, G, ipiv), n))
        A = oracle.spd_gram(n, 0)
        c, info = oracle.lapack_spotrf(A)
        arrays[f"potrf_info_{n}"] = np.int32(info)
        arrays[f"potrf_scaled_{n}"] = np.float64(oracle.scaled(oracle.potrf_residual_blas(c, A), n))
    np.savez_compressed(os.path.join(HERE, "lapack_f32.npz"), **arrays)
    print(f"{len(out)} residual cases, {len(LAPACK_N)} LAPACK sizes")


if __name__ == "__main__":
    main()
