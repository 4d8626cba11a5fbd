"""CPU tests of the C-ABI boundary: the library loads without a GPU and exports
every function that include/**/*.h declares (no compute calls)."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DECL = re.compile(
    r"^\s*(?:void|int|size_t|hdbf_status|const char\s*\*|unsigned long long)\s+\**\s*([A-Za-z_]\w*)\s*\(",
    re.M)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "**", "*.h"), recursive=True):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        names.update(DECL.findall(src))
    return sorted(names)


def test_headers_declare_reference_entry_points():
    names = set(declared_functions())
    for must in ("double_blocked_potrf", "double_blocked_potrf_kblocked_syrk",
                 "double_blocked_getrf", "double_blocked_getrf_batched_pivot",
                 "recursive_potrf", "trsm_right_lower_transpose", "gemm_nt_update",
                 "syrk_lower_update_kblocked", "launch_apply_getrf_permutation"):
        assert must in names


# Every function the reference declares under include/ (potrf, getrf, syrk,
# trsm, gemm, kernels; benchmark and utility headers excluded), FP32 and the
# `_double` twins: the drop-in boundary must declare each one.
REFERENCE_ENTRY_POINTS = (
    "batched_syrk_bottom_up", "batched_syrk_bottom_up_double", "batched_syrk_bottom_up_mixed",
    "blocked_right_looking_getrf", "blocked_right_looking_getrf_double",
    "blocked_right_looking_getrf_npvt", "blocked_right_looking_getrf_npvt_double",
    "blocked_right_looking_potrf", "blocked_right_looking_potrf_double",
    "double_blocked_getrf", "double_blocked_getrf_batched_pivot",
    "double_blocked_getrf_double", "double_blocked_getrf_double_batched_pivot",
    "double_blocked_getrf_npvt", "double_blocked_getrf_npvt_double", "double_blocked_potrf",
    "double_blocked_potrf_dbtrsm", "double_blocked_potrf_double",
    "double_blocked_potrf_double_dbtrsm", "double_blocked_potrf_double_kblocked_syrk",
    "double_blocked_potrf_double_kblocked_syrk_adaptive_gemm",
    "double_blocked_potrf_double_kblocked_syrk_adaptive_gemm_configured",
    "double_blocked_potrf_kblocked_syrk", "double_blocked_potrf_kblocked_syrk_adaptive_gemm",
    "double_blocked_potrf_kblocked_syrk_adaptive_gemm_configured", "double_blocked_trsm",
    "double_blocked_trsm_double", "gemm_nt_update", "gemm_nt_update_double",
    "gemm_nt_update_m_tiled", "gemm_nt_update_m_tiled_double", "iterative_trsm_right_looking",
    "launch_add_damping", "launch_add_damping_double", "launch_apply_getrf_panel_pivots",
    "launch_apply_getrf_panel_pivots_double", "launch_apply_getrf_permutation",
    "launch_apply_getrf_permutation_double", "launch_auto_scale", "launch_fp16_to_fp32",
    "launch_fp32_to_fp16", "launch_mixed_gemm", "recursive_potrf", "recursive_potrf_double",
    "recursive_potrf_mixed_driver", "recursive_potrf_tiled_trsm", "recursive_syrk_parallel",
    "recursive_syrk_parallel_double", "recursive_trsm", "recursive_trsm_double",
    "recursive_trsm_mixed", "recursive_trsm_tiled_update", "syrk_lower_update",
    "syrk_lower_update_double", "syrk_lower_update_kblocked",
    "syrk_lower_update_kblocked_double", "trsm_right_lower_transpose",
    "trsm_right_lower_transpose_double",
)


def test_headers_declare_every_reference_entry_point():
    names = set(declared_functions())
    missing = [n for n in REFERENCE_ENTRY_POINTS if n not in names]
    assert not missing, missing


def test_library_exports_every_declared_symbol():
    import hygondoubleblockedfactorizations_b200 as hd
    L = hd.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_exports_are_extern_c():
    lib = os.path.join(ROOT, "hygondoubleblockedfactorizations_b200", "libhdbf.so")
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    syms = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for n in declared_functions():
        assert n in syms, n  # unmangled C symbol


def test_python_prototypes_cover_headers():
    import hygondoubleblockedfactorizations_b200 as hd
    missing = set(declared_functions()) - set(hd.exported_names())
    assert not missing, missing


def test_no_oracle_in_product_sources():
    """The product (package + CUDA sources) never imports or links the oracle."""
    pkg = os.path.join(ROOT, "hygondoubleblockedfactorizations_b200")
    for f in glob.glob(os.path.join(pkg, "**", "*.*"), recursive=True):
        if f.endswith((".py", ".cu", ".h", ".cuh", ".cpp")):
            txt = open(f).read()
            assert "import oracle" not in txt and "from oracle" not in txt, f
            assert "liboracle" not in txt, f
