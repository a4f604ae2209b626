"""ctypes binding of the C ABI in include/feffgpu_b200.h (the in-tree ``_build/libfeffgpu_b200.so``).

The library is the product: there is no Python or CPU fallback.  Loading fails loudly when the shared object is
missing and cannot be built, and every call's status is turned into the exception the reference raises for the
same condition (ValueError, NotImplementedError) or RuntimeError for CUDA errors.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_build" / "libfeffgpu_b200.so"
# a different build of the same library (e.g. one compiled with other launch bounds) may be named here
if os.environ.get("FEFFGPU_B200_LIB"):
    LIB_PATH = Path(os.environ["FEFFGPU_B200_LIB"]).resolve()

FG_OK, FG_ERR_VALUE, FG_ERR_NOT_IMPLEMENTED, FG_ERR_CUDA, FG_ERR_WORKSPACE = range(5)
FG_MIXED, FG_FP64 = 0, 1
NOALLOC_SCRATCH_BYTES = 32 << 20    # FG_NOALLOC_SCRATCH_BYTES of include/feffgpu_b200.h

# every entry point of include/feffgpu_b200.h
EXPORTS = ("fg_stage_create", "fg_stage_destroy", "fg_stage_get_info", "fg_stage_lmax", "fg_stage_xk",
           "fg_last_error", "fg_cchi", "fg_cchi_backward_workspace", "fg_cchi_backward", "fg_chi_fine",
           "fg_chi_fine_backward", "fg_chi_reduce_workspace", "fg_chi_reduce", "fg_chi_reduce_noalloc",
           "fg_chi_reduce_backward_workspace",
           "fg_chi_reduce_backward", "fg_set_kernel_timing", "fg_kernel_time_ms", "fg_fp32_fma_peak", "fg_set_launch",
           "fg_stage_set_launch", "fg_stage_set_fused_variant", "fg_pf_candidates", "fg_pf_extend", "fg_pf_terminal", "fg_pf_describe",
           "fg_pf_windows", "fg_pair_histogram", "fg_pair_ss_grad", "fg_rspace_misfit",
           "fg_path_columns", "fg_chi_reduce_words", "fg_rows_from_words", "fg_path_geometry", "fg_path_geometry_backward", "fg_shard_lpt", "fg_pf_enumerate_one", "fg_pf_result_gather", "fg_pf_result_destroy")


class PhaseDesc(C.Structure):
    _fields_ = [("ne1", C.c_int32), ("nph", C.c_int32), ("ltot", C.c_int32), ("nsp", C.c_int32),
                ("ihole", C.c_int32), ("iorder", C.c_int32), ("edge", C.c_double), ("lmax0", C.c_void_p),
                ("em", C.c_void_p), ("eref", C.c_void_p), ("ph", C.c_void_p), ("rkk", C.c_void_p)]


class StageInfo(C.Structure):
    _fields_ = [("E", C.c_int32), ("L1", C.c_int32), ("nph", C.c_int32), ("kinit", C.c_int32), ("ilinit", C.c_int32),
                ("lamx_ss", C.c_int32), ("laml0x_ss", C.c_int32), ("lamx_ms", C.c_int32), ("laml0x_ms", C.c_int32),
                ("device", C.c_int32)]


class Paths(C.Structure):
    _fields_ = [("n", C.c_int64), ("nleg_max", C.c_int32), ("nrows", C.c_int32), ("coords", C.c_void_p),
                ("ipots", C.c_void_p), ("nleg", C.c_void_p), ("deg", C.c_void_p), ("sigma2", C.c_void_p),
                ("row", C.c_void_p), ("order", C.c_void_p)]


class PfTables(C.Structure):
    _fields_ = [("E", C.c_int32), ("nph1", C.c_int32), ("ik0", C.c_int32), ("fbeta", C.c_void_p),
                ("cksp", C.c_void_p), ("xlam", C.c_void_p), ("trap", C.c_void_p)]


_P = C.c_void_p
_SIGS = {
    "fg_stage_create": (C.c_int, [C.POINTER(PhaseDesc), C.c_int, C.POINTER(C.c_void_p)]),
    "fg_stage_destroy": (None, [_P]),
    "fg_stage_get_info": (C.c_int, [_P, C.POINTER(StageInfo)]),
    "fg_stage_lmax": (C.c_int, [_P, _P]),
    "fg_stage_xk": (C.c_int, [_P, _P]),
    "fg_last_error": (C.c_char_p, []),
    "fg_cchi": (C.c_int, [_P, C.c_int, C.c_int64, C.c_int32, _P, C.c_int32, _P, _P, _P, _P, _P]),
    "fg_cchi_backward_workspace": (C.c_size_t, [_P, C.c_int64, C.c_int32]),
    "fg_cchi_backward": (C.c_int, [_P, C.c_int, C.c_int64, C.c_int32, _P, C.c_int32, _P, _P, _P, _P, _P, C.c_size_t,
                                   _P]),
    "fg_chi_fine": (C.c_int, [_P, C.c_int, C.c_int64, _P, _P, C.c_int32, _P, _P, _P, _P, _P]),
    "fg_chi_fine_backward": (C.c_int, [_P, C.c_int, C.c_int64, _P, _P, C.c_int32, _P, _P, _P, _P, _P, _P, _P, _P]),
    "fg_chi_reduce_workspace": (C.c_size_t, [_P, C.POINTER(Paths), C.c_int32]),
    "fg_chi_reduce": (C.c_int, [_P, C.c_int, C.POINTER(Paths), C.c_int32, _P, _P, _P, _P, _P, _P, _P, C.c_size_t, _P]),
    "fg_chi_reduce_noalloc": (C.c_int, [_P, C.c_int, C.POINTER(Paths), C.c_int32, _P, _P, _P, _P, _P]),
    "fg_chi_reduce_backward_workspace": (C.c_size_t, [_P, C.POINTER(Paths), C.c_int32]),
    "fg_chi_reduce_backward": (C.c_int, [_P, C.c_int, C.POINTER(Paths), C.c_int32, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                         _P, C.c_size_t, _P]),
    "fg_set_kernel_timing": (C.c_int, [C.c_int32]),
    "fg_kernel_time_ms": (C.c_int, [C.POINTER(C.c_float)]),
    "fg_fp32_fma_peak": (C.c_int, [C.POINTER(C.c_double), _P]),
    "fg_set_launch": (C.c_int, [C.c_int32, C.c_int32]),
    "fg_stage_set_launch": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "fg_stage_set_fused_variant": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "fg_pf_candidates": (C.c_int, [_P, C.c_int64, C.c_float, _P, _P, C.c_int32, C.c_int32, C.c_float, _P, _P, _P,
                                   _P, _P]),
    "fg_pf_extend": (C.c_int, [C.c_int64, C.c_int32, _P, _P, _P, _P, _P, C.c_float, _P, _P, _P, _P, _P, _P]),
    "fg_pf_terminal": (C.c_int, [C.c_int64, C.c_int32, _P, _P, _P, _P, _P, _P]),
    "fg_pf_describe": (C.c_int, [C.c_int64, C.c_int32, _P, _P, _P, _P, _P, _P, _P, C.POINTER(PfTables), _P, _P, _P,
                                 _P, _P, _P, _P]),
    "fg_pf_windows": (C.c_int, [_P, _P, C.c_int64, C.c_float, _P]),
    "fg_pair_histogram": (C.c_int, [_P, C.c_int32, C.c_int64, C.c_double, _P, _P, C.c_int32, _P, C.c_int32,
                                    C.c_double, C.c_double, C.c_int32, C.c_double, _P, _P, _P]),
    "fg_pair_ss_grad": (C.c_int, [_P, C.c_int32, C.c_int64, C.c_double, _P, _P, C.c_int32, _P, C.c_double,
                                  C.c_double, C.c_int32, C.c_double, C.c_double, _P, _P]),
    "fg_rspace_misfit": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, _P, _P, _P, C.c_double, _P, _P, _P]),
    "fg_path_columns": (C.c_int, [C.c_int64, C.c_int32, C.c_int, _P, _P, _P, _P, _P, _P]),
    "fg_chi_reduce_words": (C.c_int, [_P, C.c_int, C.POINTER(Paths), C.c_int32, _P, _P, _P, _P, _P, _P, _P,
                                      C.c_size_t, _P]),
    "fg_rows_from_words": (C.c_int, [C.c_int64, C.c_int32, _P, _P, _P]),
    "fg_path_geometry": (C.c_int, [C.c_int64, C.c_int32, _P, _P, _P, _P, _P]),
    "fg_path_geometry_backward": (C.c_int, [C.c_int64, C.c_int32, _P, _P, _P, _P, _P, _P]),
    "fg_shard_lpt": (C.c_int, [_P, C.c_int64, C.c_int32, _P]),
    "fg_pf_enumerate_one": (C.c_int, [_P, C.c_int64, C.c_float, _P, C.c_int64, _P, C.POINTER(PfTables), C.c_float,
                                      C.c_int32, C.c_float, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_float), _P]),
    "fg_pf_result_gather": (C.c_int, [_P, C.c_int32, _P, _P, _P, _P, _P, _P]),
    "fg_pf_result_destroy": (None, [_P]),
}

_lock = threading.Lock()
_lib = None


def load(build_if_missing: bool = True):
    """The loaded library (built from csrc/ with nvcc first if the shared object is absent)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            if not build_if_missing:
                raise RuntimeError(f"feffgpu_b200: the CUDA library {LIB_PATH} is missing (run python -m feffgpu_b200.build)")
            from .build import build
            build()
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status: int) -> None:
    if status == FG_OK:
        return
    msg = (_lib.fg_last_error() or b"").decode(errors="replace")
    if status == FG_ERR_VALUE and msg.startswith("potential index"):
        raise IndexError(msg)                    # the reference's table lookup (stage.py:244) raises IndexError
    if status in (FG_ERR_VALUE, FG_ERR_WORKSPACE):
        raise ValueError(msg)
    if status == FG_ERR_NOT_IMPLEMENTED:
        raise NotImplementedError(msg)
    raise RuntimeError(f"feffgpu_b200: {msg}")
