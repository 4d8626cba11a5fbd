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


# --- prototypes against the reference's (tests/golden/reference_prototypes.json)
# Documented substitutions: rocblas_handle is this library's handle
# (hdbf/rocblas_compat.h), hipStream_t is cudaStream_t, __half buffers travel
# as void* (include/kernels/fp16_convert.h); every other type is unchanged.
SUBST = {"hipStream_t": "cudaStream_t", "__half*": "void*", "const __half*": "const void*"}


def _reference_prototypes():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_prototypes.json")) as f:
        return json.load(f)


def _our_prototypes():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_prototypes", os.path.join(ROOT, "tests", "golden", "make_prototypes.py"))
    mp = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mp)
    out = {}
    for h in glob.glob(os.path.join(ROOT, "include", "**", "*.h"), recursive=True):
        out.update(mp.prototypes(h))
    return out


def test_prototypes_match_reference_types():
    """A C++ translation unit includes every header through rocblas_compat.h
    and static_asserts that each entry point's type is the reference
    prototype's type after the documented substitutions (argument count,
    order and types; return type)."""
    import shutil
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    ref = _reference_prototypes()
    lines = ["#include <type_traits>", "#include \"hdbf/rocblas_compat.h\""]
    for h in sorted(glob.glob(os.path.join(ROOT, "include", "**", "*.h"), recursive=True)):
        lines.append(f'#include "{os.path.relpath(h, os.path.join(ROOT, "include"))}"')
    for name, p in sorted(ref.items()):
        types = ", ".join(SUBST.get(t, t) for t, _ in p["params"])
        lines.append(f"static_assert(std::is_same<decltype(&{name}), {p['ret']} (*)({types})>::value,"
                     f' "{name}: {p["file"]}:{p["line"]}");')
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "abi_check.cpp")
        with open(src, "w") as f:
            f.write("\n".join(lines) + "\n")
        r = subprocess.run([cxx, "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                            "-I", "/usr/local/cuda/include", src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_prototypes_match_reference_parameter_names():
    """Same parameter names in the same order as the reference (catches two
    same-typed arguments swapped, which the type check cannot)."""
    ref, ours = _reference_prototypes(), _our_prototypes()
    bad = []
    for name, p in ref.items():
        assert name in ours, name
        want = [n for _, n in p["params"]]
        got = [n for _, n in ours[name]["params"]]
        if want != got:
            bad.append((name, want, got))
    assert not bad, bad
