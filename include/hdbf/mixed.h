/*
 * Mixed-precision factorizations and FP64 iterative refinement.
 *
 * No counterpart in the reference beyond its FP16 recursive Cholesky
 * (include/potrf/recursive_potrf.h:31-37): these entry points factor with FP32
 * panels and tensor-core (tcgen05, BF16 or FP16) trailing updates that
 * accumulate in FP32 directly into the FP32 matrix, solve with the FP32
 * factors, and refine the solution of A x = b with FP64 residuals until the
 * FP64 normwise backward error max_j ||b_j - A x_j||_inf /
 * (||A||_inf ||x_j||_inf + ||b_j||_inf) reaches the requested tolerance.
 * All matrices are column-major DEVICE arrays; the refinement drivers
 * synchronise the handle's stream once per iteration to test convergence.
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hdbf_precision {
    HDBF_PREC_FP32 = 0,   /* FP32 SIMT updates (no tensor cores) */
    HDBF_PREC_BF16 = 1,   /* one BF16 product per update */
    HDBF_PREC_FP16 = 2,   /* one FP16 product per update (power-of-two operand scaling) */
    HDBF_PREC_BF16X3 = 3, /* operands split hi+lo in BF16: hi*hi + hi*lo + lo*hi */
    HDBF_PREC_FP16X3 = 4  /* operands split hi+lo in FP16 */
} hdbf_precision;

/* Right-looking block-nb factorizations with FP32 panels and trailing updates
 * in `prec`; info as the FP32 routines (first failing column, 1-based).
 * FP16 shadows carry a power-of-two scale per panel, computed on the device
 * from the panel's max |x| (no host synchronisation).  Cholesky panel
 * fallback (BF16 and FP16 modes): when a diagonal block meets a non-positive
 * pivot after the low-precision trailing updates, that panel's block column
 * is rebuilt in FP32 from a device copy of the original matrix (FP32 GEMM of
 * the preceding panels) and factored again; info is set only if the FP32
 * panel fails too.  hdbf_mixed_fallback_panels reports how many panels of the
 * handle's last mixed Cholesky took the fallback (synchronises the stream). */
hdbf_status hdbf_spotrf_mixed(hdbf_handle handle, hdbf_precision prec, float* A, int lda, int n,
                              int nb, int* info);
hdbf_status hdbf_mixed_fallback_panels(hdbf_handle handle, int* count);
hdbf_status hdbf_sgetrf_mixed(hdbf_handle handle, hdbf_precision prec, float* A, int lda, int n,
                              int nb, int* ipiv, int* info);

/* Solves with FP32 factors: B (n x nrhs) <- A^{-1} B. */
hdbf_status hdbf_spotrs(hdbf_handle handle, const float* L, int lda, int n, int nrhs, float* B,
                        int ldb);
hdbf_status hdbf_sgetrs(hdbf_handle handle, const float* LU, int lda, int n, const int* ipiv,
                        int nrhs, float* B, int ldb);

#define HDBF_IR_HISTORY 64

typedef struct hdbf_ir_info {
    int iterations;           /* refinement steps taken (residual evaluations - 1) */
    int converged;            /* 1 when backward_error <= tol */
    int final_precision;      /* hdbf_precision of the factors that were used */
    int factorizations;       /* 1 + escalations */
    int info;                 /* info of the last factorization */
    double backward_error;    /* final FP64 normwise backward error (max over columns) */
    double history[HDBF_IR_HISTORY]; /* backward error after each step (history[0] = initial) */
    double factor_ms;         /* device time of the factorizations */
    double refine_ms;         /* device time of solves + residuals + updates */
    int inner_iterations;     /* GMRES-IR: preconditioned GMRES steps over all outer steps */
    int fallback_panels;      /* Cholesky panels rebuilt in FP32 by the last factorization */
} hdbf_ir_info;

/* Solve A X = B (A SPD for posv, general for gesv; A, B, X FP64).  The FP64 A
 * is rounded to an FP32 working copy that is factored with `prec`; classical
 * refinement x += A^{-1}(b - A x) runs with FP64 residuals.  With `escalate`,
 * a step that does not halve the backward error (or a failed factorization)
 * refactors at the next precision (BF16 -> BF16X3 -> FP32, FP16 -> FP16X3 ->
 * FP32); the first step with the new factors is taken without that test.
 * nrhs <= 64.  X may alias nothing else. */
hdbf_status hdbf_dposv_mixed(hdbf_handle handle, hdbf_precision prec, int escalate,
                             const double* A, int lda, int n, int nrhs, const double* B, int ldb,
                             double* X, int ldx, double tol, int max_iter, hdbf_ir_info* out);
hdbf_status hdbf_dgesv_mixed(hdbf_handle handle, hdbf_precision prec, int escalate,
                             const double* A, int lda, int n, int nrhs, const double* B, int ldb,
                             double* X, int ldx, double tol, int max_iter, hdbf_ir_info* out);

/* GMRES-IR (Carson-Higham): the same factorizations, but each correction
 * solves A d = r with restarted GMRES in FP64 (at most max_inner steps, CGS2
 * orthogonalisation, all right-hand sides in lockstep) preconditioned from the
 * left by the low-precision factors, until the preconditioned residual falls
 * by inner_tol.  Converges where classical refinement stalls (BF16/FP16 LU of
 * large n, or kappa * u_factor near or above 1).  Outer steps stop at tol or
 * max_iter; no escalation.  nrhs <= 64. */
hdbf_status hdbf_dposv_mixed_gmres(hdbf_handle handle, hdbf_precision prec, const double* A,
                                   int lda, int n, int nrhs, const double* B, int ldb, double* X,
                                   int ldx, double tol, int max_iter, int max_inner,
                                   double inner_tol, hdbf_ir_info* out);
hdbf_status hdbf_dgesv_mixed_gmres(hdbf_handle handle, hdbf_precision prec, const double* A,
                                   int lda, int n, int nrhs, const double* B, int ldb, double* X,
                                   int ldx, double tol, int max_iter, int max_inner,
                                   double inner_tol, hdbf_ir_info* out);

/* Adaptive refinement: one call that picks the refinement and, if needed, a
 * higher factorization precision.
 *  - Classical corrections d = M^{-1} r while each at least halves the
 *    backward error.
 *  - From the first that does not, GMRES-IR steps (30 inner steps, inner
 *    tolerance 1e-4) on the same factors.
 *  - When a GMRES step does not halve the backward error, or the steps still
 *    needed at its rate would take longer than two factorizations (device
 *    times measured during the call), the matrix is refactored at the next
 *    precision (BF16 -> BF16x3 -> FP32, FP16 -> FP16x3 -> FP32; also when the
 *    factorization itself fails).  Classical corrections with the new factors
 *    continue from the current solution (the first one is not judged), again
 *    until they stall.
 *  - hdbf_dgesv_mixed_auto with BF16 or FP16 skips the GMRES stage on those
 *    single-word factors: when their classical corrections stall it refactors
 *    with the FP16 split (FP16x3) at once, from BF16 too (22 significant bits
 *    against BF16x3's 16, at the same cost).
 * Stops at tol or after max_iter outer steps; out->final_precision and
 * out->factorizations record the escalations.  nrhs <= 64. */
hdbf_status hdbf_dposv_mixed_auto(hdbf_handle handle, hdbf_precision prec, const double* A,
                                  int lda, int n, int nrhs, const double* B, int ldb, double* X,
                                  int ldx, double tol, int max_iter, hdbf_ir_info* out);
hdbf_status hdbf_dgesv_mixed_auto(hdbf_handle handle, hdbf_precision prec, const double* A,
                                  int lda, int n, int nrhs, const double* B, int ldb, double* X,
                                  int ldx, double tol, int max_iter, hdbf_ir_info* out);

#ifdef __cplusplus
}
#endif
