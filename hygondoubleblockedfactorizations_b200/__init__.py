"""B200-native double-blocked dense factorizations (host-side Python binding).

The product is ``libhdbf.so`` (CUDA kernels for sm_100a + C++ host drivers
behind a C ABI whose entry points mirror the reference's ``include/`` tree).
This module only loads that library with ``ctypes`` and exposes the same
functions with the same names and argument order; device memory is passed as
raw pointers (``torch.Tensor.data_ptr()`` works).  There is no fallback: if the
library is missing, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libhdbf.so")

_lib = None

c_int, c_float, c_double = ctypes.c_int, ctypes.c_float, ctypes.c_double
c_void_p, c_size_t, c_ull = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_ulonglong
P = c_void_p  # every device pointer travels as void*

# name -> (restype, argtypes)
_PROTOS = {
    # runtime (include/hdbf/hdbf.h)
    "hdbf_create": (c_int, [ctypes.POINTER(c_void_p)]),
    "hdbf_destroy": (c_int, [P]),
    "hdbf_set_stream": (c_int, [P, P]),
    "hdbf_get_stream": (c_int, [P, ctypes.POINTER(c_void_p)]),
    "hdbf_get_last_status": (c_int, [P]),
    "hdbf_status_string": (ctypes.c_char_p, [c_int]),
    "hdbf_reserve_workspace": (c_int, [P, c_size_t]),
    "hdbf_workspace_bytes_for": (c_size_t, [c_int]),
    "hdbf_check_device_errors": (c_int, [P]),
    "hdbf_stream_pool_create": (c_int, [c_int, ctypes.POINTER(c_void_p)]),
    "hdbf_stream_pool_destroy": (c_int, [P]),
    "hdbf_stream_pool_size": (c_int, [P]),
    "hdbf_fill_uniform": (c_int, [P, P, c_size_t, c_ull, c_ull]),
    "hdbf_launch_count": (c_ull, [P]),
    "hdbf_profile_begin": (c_int, [P]),
    "hdbf_profile_end": (c_int, [P, c_int, P, P, P, P]),
    "hdbf_profile_class_name": (ctypes.c_char_p, [c_int]),
    "hdbf_profile_num_classes": (c_int, []),
    "hdbf_profile_num_stages": (c_int, []),
    "hdbf_profile_stage_name": (ctypes.c_char_p, [c_int]),
    "hdbf_profile_stages": (c_int, [P, c_int, P, P, P]),
    "hdbf_set_graph_mode": (c_int, [P, c_int]),
    "hdbf_set_panel_kernel": (c_int, [P, c_int]),
    "hdbf_set_lookahead": (c_int, [P, c_int]),
    "hdbf_set_wait_limit": (c_int, [P, ctypes.c_uint]),
    "hdbf_mixed_fallback_panels": (c_int, [P, ctypes.POINTER(c_int)]),
    # potrf
    "double_blocked_potrf": (None, [P, P, c_int, c_int, c_int, c_int, P]),
    "double_blocked_potrf_dbtrsm": (None, [P, P, c_int, c_int, c_int, c_int, P]),
    "double_blocked_potrf_kblocked_syrk": (None, [P, P, c_int, c_int, c_int, c_int, c_int, P]),
    "double_blocked_potrf_kblocked_syrk_adaptive_gemm":
        (None, [P, P, c_int, c_int, c_int, c_int, c_int, P]),
    "double_blocked_potrf_kblocked_syrk_adaptive_gemm_configured":
        (None, [P, P, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int, P]),
    "blocked_right_looking_potrf": (None, [P, P, c_int, c_int, c_int, P]),
    "recursive_potrf": (None, [P, P, P, c_int, c_int, c_int, P]),
    "recursive_potrf_tiled_trsm": (None, [P, P, P, c_int, c_int, c_int, P]),
    # getrf
    "double_blocked_getrf": (None, [P, P, c_int, c_int, c_int, c_int, c_int, c_int, P, P]),
    "double_blocked_getrf_batched_pivot":
        (None, [P, P, c_int, c_int, c_int, c_int, c_int, c_int, c_int, P, P, P]),
    "double_blocked_getrf_npvt": (None, [P, P, c_int, c_int, c_int, c_int, P]),
    "blocked_right_looking_getrf": (None, [P, P, c_int, c_int, c_int, P, P]),
    "blocked_right_looking_getrf_npvt": (None, [P, P, c_int, c_int, c_int, P]),
    "launch_apply_getrf_panel_pivots": (None, [P, c_int, c_int, c_int, c_int, P, P]),
    "launch_apply_getrf_permutation": (None, [P, c_int, c_int, P, P, c_int, P, c_int, P]),
    # syrk / trsm / gemm
    "syrk_lower_update": (None, [P, c_int, c_int, P, c_int, P, c_int]),
    "syrk_lower_update_kblocked": (None, [P, c_int, c_int, P, c_int, P, c_int, c_int]),
    "recursive_syrk_parallel": (None, [P, P, c_int, P, c_int, c_int, c_int, c_int]),
    "batched_syrk_bottom_up": (None, [P, P, P, c_int, P, c_int, c_int, c_int, c_int]),
    "trsm_right_lower_transpose": (None, [P, c_int, c_int, P, c_int, P, c_int]),
    "trsm_right_lower_transpose_noalloc": (c_int, [c_int, c_int, P, c_int, P, c_int, P]),
    "double_blocked_trsm": (None, [P, P, c_int, P, c_int, c_int, c_int, c_int, c_int]),
    "recursive_trsm": (None, [P, P, c_int, P, c_int, c_int, c_int, c_int]),
    "recursive_trsm_tiled_update": (None, [P, P, c_int, P, c_int, c_int, c_int, c_int]),
    "iterative_trsm_right_looking": (None, [P, P, c_int, P, c_int, c_int, c_int, c_int]),
    "gemm_nt_update": (None, [P, c_int, c_int, c_int, P, c_int, P, c_int, P, c_int]),
    "gemm_nt_update_m_tiled": (None, [P, c_int, c_int, c_int, P, c_int, P, c_int, P, c_int, c_int]),
    "recursive_potrf_mixed_driver": (None, [P, P, P, c_int, c_int, c_int, P]),
    "batched_syrk_bottom_up_mixed": (None, [P, P, P, c_int, P, c_int, c_int, c_int, c_int]),
    "recursive_trsm_mixed": (None, [P, P, c_int, P, c_int, c_int, c_int, c_int]),
    "hdbf_spotrf_mixed": (c_int, [P, c_int, P, c_int, c_int, c_int, P]),
    "hdbf_sgetrf_mixed": (c_int, [P, c_int, P, c_int, c_int, c_int, P, P]),
    "hdbf_spotrs": (c_int, [P, P, c_int, c_int, c_int, P, c_int]),
    "hdbf_sgetrs": (c_int, [P, P, c_int, c_int, P, c_int, P, c_int]),
    "hdbf_dposv_mixed": (c_int, [P, c_int, c_int, P, c_int, c_int, c_int, P, c_int, P, c_int,
                                 c_double, c_int, P]),
    "hdbf_dgesv_mixed": (c_int, [P, c_int, c_int, P, c_int, c_int, c_int, P, c_int, P, c_int,
                                 c_double, c_int, P]),
    "hdbf_dposv_mixed_gmres": (c_int, [P, c_int, P, c_int, c_int, c_int, P, c_int, P, c_int,
                                       c_double, c_int, c_int, c_double, P]),
    "hdbf_dgesv_mixed_gmres": (c_int, [P, c_int, P, c_int, c_int, c_int, P, c_int, P, c_int,
                                       c_double, c_int, c_int, c_double, P]),
    "hdbf_dposv_mixed_auto": (c_int, [P, c_int, P, c_int, c_int, c_int, P, c_int, P, c_int,
                                      c_double, c_int, P]),
    "hdbf_dgesv_mixed_auto": (c_int, [P, c_int, P, c_int, c_int, c_int, P, c_int, P, c_int,
                                      c_double, c_int, P]),
    "hdbf_selector_num_params": (c_int, [c_int, c_int]),
    "hdbf_selector_init": (c_int, [P, P, c_int, c_int, c_ull]),
    "hdbf_selector_train": (c_int, [P, P, P, P, c_int, P, P, P, c_int, c_int, c_int, c_int,
                                    c_float, c_float, P, P]),
    "hdbf_selector_predict": (c_int, [P, P, P, P, c_int, c_int, c_int, P, P, P]),
    "hdbf_batched_num_variants": (c_int, []),
    "hdbf_batched_variant_shape": (c_int, [c_int, P, P]),
    "hdbf_batched_factor_solve": (c_int, [P, c_int, c_int, P, P, P, P, P, P, P, P, P]),
    "launch_mixed_gemm": (None, [P, P, c_int, c_int, c_int, c_int, c_int, c_float, P, c_int, P,
                                 c_int, c_float, P, c_int]),
    # FP64 twins (the reference's `_double` entry points)
    "double_blocked_potrf_double": (None, [P, P, c_int, c_int, c_int, c_int, P]),
    "double_blocked_potrf_double_dbtrsm": (None, [P, P, c_int, c_int, c_int, c_int, P]),
    "double_blocked_potrf_double_kblocked_syrk":
        (None, [P, P, c_int, c_int, c_int, c_int, c_int, P]),
    "double_blocked_potrf_double_kblocked_syrk_adaptive_gemm":
        (None, [P, P, c_int, c_int, c_int, c_int, c_int, P]),
    "double_blocked_potrf_double_kblocked_syrk_adaptive_gemm_configured":
        (None, [P, P, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int, P]),
    "blocked_right_looking_potrf_double": (None, [P, P, c_int, c_int, c_int, P]),
    "recursive_potrf_double": (None, [P, P, P, c_int, c_int, c_int, P]),
    "double_blocked_getrf_double":
        (None, [P, P, c_int, c_int, c_int, c_int, c_int, c_int, P, P]),
    "double_blocked_getrf_double_batched_pivot":
        (None, [P, P, c_int, c_int, c_int, c_int, c_int, c_int, c_int, P, P, P]),
    "double_blocked_getrf_npvt_double": (None, [P, P, c_int, c_int, c_int, c_int, P]),
    "blocked_right_looking_getrf_double": (None, [P, P, c_int, c_int, c_int, P, P]),
    "blocked_right_looking_getrf_npvt_double": (None, [P, P, c_int, c_int, c_int, P]),
    "launch_apply_getrf_panel_pivots_double": (None, [P, c_int, c_int, c_int, c_int, P, P]),
    "launch_apply_getrf_permutation_double":
        (None, [P, c_int, c_int, P, P, c_int, P, c_int, P]),
    "syrk_lower_update_double": (None, [P, c_int, c_int, P, c_int, P, c_int]),
    "syrk_lower_update_kblocked_double": (None, [P, c_int, c_int, P, c_int, P, c_int, c_int]),
    "recursive_syrk_parallel_double": (None, [P, P, c_int, P, c_int, c_int, c_int, c_int]),
    "batched_syrk_bottom_up_double": (None, [P, P, P, c_int, P, c_int, c_int, c_int, c_int]),
    "trsm_right_lower_transpose_double": (None, [P, c_int, c_int, P, c_int, P, c_int]),
    "double_blocked_trsm_double": (None, [P, P, c_int, P, c_int, c_int, c_int, c_int, c_int]),
    "recursive_trsm_double": (None, [P, P, c_int, P, c_int, c_int, c_int, c_int]),
    "gemm_nt_update_double": (None, [P, c_int, c_int, c_int, P, c_int, P, c_int, P, c_int]),
    "gemm_nt_update_m_tiled_double":
        (None, [P, c_int, c_int, c_int, P, c_int, P, c_int, P, c_int, c_int]),
    # kernels
    "launch_add_damping": (None, [P, c_int, c_int, c_float, P]),
    "launch_add_damping_double": (None, [P, c_int, c_int, c_double, P]),
    "launch_fp32_to_fp16": (None, [P, P, c_int, c_int, c_int, c_int, P]),
    "launch_fp16_to_fp32": (None, [P, P, c_int, c_int, c_int, c_int, P]),
    "launch_auto_scale": (None, [P, c_int, c_int, P, ctypes.c_bool, P]),
}


PREC = {"fp32": 0, "bf16": 1, "fp16": 2, "bf16x3": 3, "fp16x3": 4}


class IrInfo(ctypes.Structure):
    """hdbf_ir_info (include/hdbf/mixed.h)."""
    _fields_ = [("iterations", c_int), ("converged", c_int), ("final_precision", c_int),
                ("factorizations", c_int), ("info", c_int), ("backward_error", c_double),
                ("history", c_double * 64), ("factor_ms", c_double), ("refine_ms", c_double),
                ("inner_iterations", c_int), ("fallback_panels", c_int)]


class HdbfError(RuntimeError):
    pass


def lib():
    """Load libhdbf.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HdbfError(f"{LIB_PATH} is missing: build it with "
                            "`python -m hygondoubleblockedfactorizations_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_names():
    return list(_PROTOS)


class WorkspacePivot(ctypes.Structure):
    """getrf_batched_pivot_workspace (include/getrf/double_blocked_getrf.h)."""
    _fields_ = [("device_sources", c_void_p), ("device_targets", c_void_p),
                ("device_swap_buffer", c_void_p), ("host_pivots", c_void_p),
                ("host_permutation", c_void_p), ("host_sources", c_void_p),
                ("host_targets", c_void_p), ("capacity", c_int), ("column_tile", c_int)]


class Handle:
    """Owns an hdbf_handle bound to a CUDA stream (an int/handle or None)."""

    def __init__(self, stream=None):
        self._h = c_void_p()
        st = lib().hdbf_create(ctypes.byref(self._h))
        if st != 0:
            raise HdbfError(f"hdbf_create failed: {status_string(st)}")
        if stream is not None:
            self.set_stream(stream)

    @property
    def ptr(self):
        return self._h

    def set_stream(self, stream):
        s = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", stream)
        lib().hdbf_set_stream(self._h, c_void_p(s))

    def last_status(self) -> int:
        return lib().hdbf_get_last_status(self._h)

    def check(self, what="call"):
        st = self.last_status()
        if st != 0:
            raise HdbfError(f"{what}: {status_string(st)}")

    def device_errors(self) -> int:
        return lib().hdbf_check_device_errors(self._h)

    def reserve(self, nbytes: int):
        st = lib().hdbf_reserve_workspace(self._h, nbytes)
        if st != 0:
            raise HdbfError(f"reserve_workspace: {status_string(st)}")

    def set_panel_kernel(self, mode: int):
        """0 automatic, 1 grid-wide publish-and-poll kernel, 2 cluster kernel."""
        st = lib().hdbf_set_panel_kernel(self._h, int(mode))
        if st != 0:
            raise HdbfError(f"set_panel_kernel: {status_string(st)}")

    def set_lookahead(self, enabled: bool):
        """Overlap the GETRF panel chain with the outer update (batched/no pivoting)."""
        st = lib().hdbf_set_lookahead(self._h, 1 if enabled else 0)
        if st != 0:
            raise HdbfError(f"set_lookahead: {status_string(st)}")

    def set_wait_limit(self, polls: int):
        """Poll limit of the bounded device-side waits (0: the default)."""
        st = lib().hdbf_set_wait_limit(self._h, int(polls))
        if st != 0:
            raise HdbfError(f"hdbf_set_wait_limit: {status_string(st)}")

    def set_graphs(self, enabled: bool):
        lib().hdbf_set_graph_mode(self._h, 1 if enabled else 0)

    def launches(self) -> int:
        return int(lib().hdbf_launch_count(self._h))

    def profile_begin(self):
        lib().hdbf_profile_begin(self._h)

    def profile_end(self):
        """Per kernel class: {name: (launches, total_ms, flops, bytes)}."""
        L = lib()
        k = L.hdbf_profile_num_classes()
        ms, fl, by = (c_double * k)(), (c_double * k)(), (c_double * k)()
        ln = (c_ull * k)()
        st = L.hdbf_profile_end(self._h, k, ms, fl, by, ln)
        if st != 0:
            raise HdbfError(f"profile_end: {status_string(st)}")
        return {L.hdbf_profile_class_name(i).decode(): (int(ln[i]), ms[i], fl[i], by[i])
                for i in range(k) if ln[i]}

    def profile_stages(self):
        """Per driver stage of the last profiling interval (stages that ran,
        in the library's stage order): {name: (calls, total_ms, flops)}."""
        L = lib()
        k = L.hdbf_profile_num_stages()
        ms, fl = (c_double * k)(), (c_double * k)()
        calls = (c_int * k)()
        st = L.hdbf_profile_stages(self._h, k, ms, fl, calls)
        if st != 0:
            raise HdbfError(f"profile_stages: {status_string(st)}")
        return {L.hdbf_profile_stage_name(i).decode(): (int(calls[i]), ms[i], fl[i])
                for i in range(1, k) if calls[i]}

    def close(self):
        if self._h:
            lib().hdbf_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def status_string(st: int) -> str:
    return lib().hdbf_status_string(st).decode()


def call(name: str, *args):
    """Call a C-ABI entry point by its reference name."""
    return getattr(lib(), name)(*args)
