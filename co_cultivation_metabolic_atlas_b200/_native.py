"""ctypes binding of the C ABI declared in ``include/fbalp.h``.

The library is loaded from the package's ``_lib`` directory (built in-tree by
``build.py``).  There is no fallback: if the library is missing or a symbol is
absent, import of the engine fails loudly.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libfbalp.so"

FBALP_OK = 0
FBALP_ERR_INVALID = 1
FBALP_ERR_CUDA = 2
FBALP_ERR_ALLOC = 3
FBALP_ERR_STATE = 4

STATUS_OPTIMAL = 0
STATUS_ITERATION_LIMIT = 1
STATUS_NUMERICAL = 2
STATUS_INVALID_INPUT = 3
STATUS_NOT_RUN = 4
STATUS_HANDOFF = 5
STATUS_NAMES = {0: "optimal", 1: "iteration_limit", 2: "numerical", 3: "invalid_input",
                4: "not_run", 5: "handoff"}

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_FP32 = 2

METRICS = 8
MAX_PATCHES = 8      # FBALP_MAX_PATCHES
METRIC_NAMES = ("primal_residual", "dual_violation", "relative_kkt_gap", "objective",
                "dual_objective", "relative_gap", "x_inf", "omega")

c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_int64_p = ctypes.POINTER(ctypes.c_int64)
c_double_p = ctypes.POINTER(ctypes.c_double)


class Options(ctypes.Structure):
    _fields_ = [("ruiz_iterations", ctypes.c_int32), ("power_iterations", ctypes.c_int32),
                ("step_safety", ctypes.c_double), ("warps_per_block", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("max_dynamic_smem", ctypes.c_int32),
                ("stage_matrix", ctypes.c_int32), ("fp64_max_dynamic_smem", ctypes.c_int32),
                ("pair_instances", ctypes.c_int32), ("spread_banks", ctypes.c_int32)]


class SolveParams(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("max_iterations", ctypes.c_int32),
                ("fp32_max_iterations", ctypes.c_int32), ("check_every", ctypes.c_int32),
                ("tol_primal", ctypes.c_double), ("tol_dual", ctypes.c_double),
                ("tol_gap", ctypes.c_double), ("fp32_tol_primal", ctypes.c_double),
                ("fp32_tol_dual", ctypes.c_double), ("fp32_tol_gap", ctypes.c_double),
                ("reflection", ctypes.c_double), ("restarts", ctypes.c_int32),
                ("fp32_stall_checks", ctypes.c_int32), ("fp64_stall_checks", ctypes.c_int32),
                ("floor_tol", ctypes.c_double), ("fp32_passthrough_tol", ctypes.c_double),
                ("fallback_iterations", ctypes.c_int32), ("fp32_recentre", ctypes.c_int32),
                ("fp32_values_phase", ctypes.c_int32), ("gate_primal", ctypes.c_double),
                ("gate_dual", ctypes.c_double), ("gate_gap", ctypes.c_double),
                ("primal_weight_smoothing", ctypes.c_double)]


KERNEL_NAMES = {-1: None, 0: "pdhg_persistent<float>", 1: "pdhg_persistent<double>", 2: "pdhg_recentred<staged>",
                3: "pdhg_recentred<streamed>", 4: "pdhg_recentred_pair", 5: "pdhg_recentred<staged, fp32 values>",
                6: "pdhg_recentred<streamed, fp32 values>"}


class NativeError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"fbalp error {code}: {message}")
        self.code = code


_lib = None


def load(path: os.PathLike | None = None):
    """Load (once) and return the native library with typed signatures."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"native library {p} is missing; run co_cultivation_metabolic_atlas_b200.build")
    lib = ctypes.CDLL(str(p))
    vp = ctypes.c_void_p
    sig = {
        "fbalp_default_options": (None, [ctypes.POINTER(Options)]),
        "fbalp_default_solve_params": (None, [ctypes.POINTER(SolveParams)]),
        "fbalp_engine_create": (ctypes.c_int, [ctypes.c_int32, c_int32_p, c_int32_p, c_int32_p,
                                               ctypes.POINTER(c_int64_p), ctypes.POINTER(c_int32_p),
                                               ctypes.POINTER(c_double_p), ctypes.POINTER(Options), vp,
                                               ctypes.POINTER(vp)]),
        "fbalp_engine_set_instances": (ctypes.c_int, [vp, ctypes.c_int64, c_int32_p, vp, vp, vp, vp]),
        "fbalp_engine_set_instance_data": (ctypes.c_int, [vp, vp, vp, vp, vp]),
        "fbalp_engine_set_iteration_hints": (ctypes.c_int, [vp, vp]),
        "fbalp_engine_set_patches": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p]),
        "fbalp_engine_set_patch_values": (ctypes.c_int, [vp, vp, ctypes.c_int32]),
        "fbalp_scaled_certificate": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                    vp, vp, vp, vp, vp, vp, ctypes.c_int32, vp, vp, vp,
                                                    vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int32, vp,
                                                    vp, vp, vp, vp]),
        "fbalp_engine_solve": (ctypes.c_int, [vp, vp, vp, vp, ctypes.POINTER(SolveParams), vp, vp, vp, vp,
                                              vp, vp, vp]),
        "fbalp_engine_destroy": (ctypes.c_int, [vp]),
        "fbalp_engine_solve_noalloc": (ctypes.c_int, [vp, ctypes.c_int64, vp, vp, vp, vp, vp, vp, vp,
                                                      ctypes.POINTER(SolveParams), vp, vp, vp, vp, vp, vp, vp]),
        "fbalp_engine_set_stream": (ctypes.c_int, [vp, vp]),
        "fbalp_engine_layout": (ctypes.c_int, [vp, c_int64_p, c_int64_p, c_int64_p, c_int64_p]),
        "fbalp_prepare_matrix": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int64_p, c_int32_p,
                                                c_double_p, ctypes.POINTER(Options), c_double_p,
                                                c_double_p, c_double_p, c_double_p]),
        "fbalp_engine_phase_times": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_float),
                                                    ctypes.POINTER(ctypes.c_float)]),
        "fbalp_engine_phase_iterations": (ctypes.c_int, [vp, vp]),
        "fbalp_engine_phase_kernels": (ctypes.c_int, [vp, c_int32_p, c_int32_p]),
        "fbalp_engine_timing_slots": (ctypes.c_int, [vp, ctypes.c_int32]),
        "fbalp_engine_use_timing_slot": (ctypes.c_int, [vp, ctypes.c_int32]),
        "fbalp_engine_slot_times": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_float),
                                                   ctypes.POINTER(ctypes.c_float)]),
        "fbalp_last_error": (ctypes.c_char_p, []),
        # BF16 tensor-core kernels of the learned warm start (include/fbalp_mlp.h)
        "fbalp_gemm_bf16": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int,
                                           ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int,
                                           ctypes.c_float, vp, vp, ctypes.c_int, vp, ctypes.c_int,
                                           ctypes.c_int, vp]),
        "fbalp_mlp_error_flag": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
        "fbalp_gelu_backward": (ctypes.c_int, [ctypes.c_int64, vp, vp, vp, vp, vp]),
        "fbalp_mse_grad": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_float, vp, vp, vp, vp]),
        "fbalp_column_sum": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, vp, vp, vp]),
        "fbalp_adam_step": (ctypes.c_int, [ctypes.c_int64, vp, vp, vp, vp, vp, ctypes.c_float, ctypes.c_float,
                                           ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float, vp]),
        "fbalp_to_bf16": (ctypes.c_int, [ctypes.c_int64, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)  # AttributeError if the symbol is missing
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code: int):
    if code != FBALP_OK:
        msg = _lib.fbalp_last_error().decode(errors="replace") if _lib else ""
        raise NativeError(code, msg)


def default_options() -> Options:
    o = Options()
    load().fbalp_default_options(ctypes.byref(o))
    return o


def default_solve_params() -> SolveParams:
    p = SolveParams()
    load().fbalp_default_solve_params(ctypes.byref(p))
    return p
