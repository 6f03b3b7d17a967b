"""ctypes binding of ``libgd_poisson.so`` (the C ABI of ``include/gd_poisson.h``).

There is no CPU fallback: importing the solvers works anywhere, but the first
call that needs the library raises if the shared object is missing, and the
first call that needs a GPU raises if CUDA is unavailable.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgd_poisson.so")

GD_DIRICHLET, GD_NEUMANN, GD_MASKED = 0, 1, 2
GD_MIXED, GD_FP64 = 0, 1
GD_CONVERGED, GD_MAX_ITERATIONS, GD_BREAKDOWN, GD_ACTIVE, GD_STAGNATED = 0, 1, 2, 3, 4
STATUS_NAMES = {0: "converged", 1: "max_iterations", 2: "breakdown", 3: "active",
                4: "stagnated"}

EXPORTS = (
    "gd_last_error", "gd_version", "gd_plan_create", "gd_plan_destroy",
    "gd_plan_workspace_bytes", "gd_plan_bind", "gd_plan_set_mask", "gd_plan_prepare",
    "gd_solve", "gd_solve_async", "gd_solve_finish", "gd_plan_apply_vcycle", "gd_plan_set_profiling", "gd_plan_kernel_times", "gd_plan_level_times",
    "gd_ref_workspace_bytes", "gd_ref_vcycle", "gd_ref_vcycle_static", "gd_rbgs_smooth",
    "gd_ref_residual", "gd_ref_dot", "gd_ref_axpby", "gd_ref_restrict", "gd_ref_prolong_add", "gd_gradient", "gd_divergence", "gd_fold_dirichlet",
    "gd_fold_boundary",
    "gd_masked_rhs", "gd_guidance_divergence", "gd_tm_scratch_bytes", "gd_tm_log_luminance",
    "gd_tm_downsample", "gd_tm_level_factor", "gd_tm_compose", "gd_dct_plan_create",
    "gd_dct_workspace_bytes", "gd_dct_plan_bind", "gd_dct_solve_neumann", "gd_dct_plan_destroy",
    "gd_selftest_bounded_wait",
)


class GridDesc(C.Structure):
    _fields_ = [("height", C.c_int32), ("width", C.c_int32), ("boundary", C.c_int32),
                ("flags", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("precision", C.c_int32), ("pre_sweeps", C.c_int32),
                ("post_sweeps", C.c_int32), ("max_iterations", C.c_int32),
                ("tolerance", C.c_double), ("reliable_delta", C.c_double),
                ("check_every", C.c_int32), ("use_graph", C.c_int32),
                ("strip_target_warps", C.c_int32), ("bottom_cells", C.c_int32),
                ("tile_cells", C.c_int32), ("zero_start", C.c_int32),
                ("persistent_coarse", C.c_int32), ("dependent_launch", C.c_int32)]


class Report(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("status", C.c_int32),
                ("relative_residual", C.c_double), ("initial_norm", C.c_double),
                ("refreshes", C.c_int32), ("reserved", C.c_int32)]


class FieldDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("height", C.c_int32), ("width", C.c_int32),
                ("channels", C.c_int32), ("channel", C.c_int32), ("edges", C.c_int32),
                ("target", C.c_void_p), ("source", C.c_void_p), ("select", C.c_void_p),
                ("weights", C.c_void_p), ("alpha_pow_beta", C.c_double), ("beta", C.c_double),
                ("epsilon", C.c_double)]


GD_FIELD_IMPORT, GD_FIELD_MIXED, GD_FIELD_AVERAGE, GD_FIELD_WEIGHTED, GD_FIELD_ILLUMINATION = \
    range(5)


class KernelTime(C.Structure):
    _fields_ = [("launches", C.c_longlong), ("milliseconds", C.c_double), ("cells", C.c_double)]


KERNEL_KINDS = ("down0", "down", "bottom", "up", "up0", "pupdate", "cgupdate", "fold", "resid",
                "init", "mean", "coarse")
PROFILE_LEVELS = 32


class GDError(RuntimeError):
    """A call into libgd_poisson failed."""


_lock = threading.Lock()
_lib: C.CDLL | None = None

_vp, _dp, _i32, _i64, _f64, _sz = C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_size_t


def _declare(lib: C.CDLL) -> None:
    sig = {
        "gd_last_error": (C.c_char_p, []),
        "gd_version": (C.c_char_p, []),
        "gd_plan_create": (C.c_int, [C.POINTER(GridDesc), _i32, C.POINTER(Params),
                                     C.POINTER(C.c_void_p)]),
        "gd_plan_destroy": (None, [_vp]),
        "gd_plan_workspace_bytes": (_sz, [_vp]),
        "gd_plan_bind": (C.c_int, [_vp, _vp, _sz, _vp]),
        "gd_plan_set_mask": (C.c_int, [_vp, _i32, _vp, _i32, _vp]),
        "gd_plan_prepare": (C.c_int, [_vp, _vp]),
        "gd_solve": (C.c_int, [_vp, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                               C.POINTER(C.c_int32), C.POINTER(C.c_double), _vp,
                               C.POINTER(Report)]),
        "gd_solve_async": (C.c_int, [_vp, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_double), _vp]),
        "gd_solve_finish": (C.c_int, [_vp, C.POINTER(Report)]),
        "gd_plan_apply_vcycle": (C.c_int, [_vp, _i32, _vp, _vp, _i32, _vp]),
        "gd_plan_set_profiling": (C.c_int, [_vp, _i32]),
        "gd_plan_kernel_times": (C.c_int, [_vp, C.POINTER(KernelTime), _i32]),
        "gd_plan_level_times": (C.c_int, [_vp, C.POINTER(KernelTime), _i32]),
        "gd_selftest_bounded_wait": (C.c_int, [_i32, _vp, _vp, _vp]),
        "gd_ref_workspace_bytes": (_sz, [_i32, _i32, _i32]),
        "gd_ref_vcycle": (C.c_int, [_vp, _vp, _i32, _i32, _f64, _i32, _i32, _i32, _i32, _vp,
                                    _sz, _vp]),
        "gd_ref_vcycle_static": (C.c_int, [_vp, _vp, _i32, _i32, _f64, _i32, _i32, _i32, _i32,
                                           _vp]),
        "gd_rbgs_smooth": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _i32, _i32, _f64, _i32, _vp]),
        "gd_ref_residual": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _f64, _vp]),
        "gd_ref_dot": (C.c_int, [_vp, _vp, _vp, _i64, _vp, _sz, _vp]),
        "gd_ref_axpby": (C.c_int, [_vp, _vp, _f64, _f64, _i64, _vp]),
        "gd_ref_restrict": (C.c_int, [_vp, _vp, _i32, _i32, _vp]),
        "gd_ref_prolong_add": (C.c_int, [_vp, _vp, _i32, _i32, _i32, _i32, _vp]),
        "gd_gradient": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _vp]),
        "gd_divergence": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _vp]),
        "gd_fold_dirichlet": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _f64, _vp]),
        "gd_fold_boundary": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _i32, _f64, _vp]),
        "gd_masked_rhs": (C.c_int, [_vp, _vp, _vp, _vp, _i32, _i32, _f64, _vp]),
        "gd_guidance_divergence": (C.c_int, [_vp, C.POINTER(FieldDesc), _i32, _i32, _i32, _i32,
                                             _vp]),
        "gd_tm_scratch_bytes": (_sz, []),
        "gd_dct_plan_create": (C.c_int, [_i32, _i32, C.POINTER(C.c_void_p)]),
        "gd_dct_workspace_bytes": (_sz, [_vp]),
        "gd_dct_plan_bind": (C.c_int, [_vp, _vp, _sz, _vp]),
        "gd_dct_solve_neumann": (C.c_int, [_vp, _vp, _vp, _i32, _vp]),
        "gd_dct_plan_destroy": (None, [_vp]),
        "gd_tm_log_luminance": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _vp]),
        "gd_tm_downsample": (C.c_int, [_vp, _vp, _i32, _i32, _vp]),
        "gd_tm_level_factor": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _i32, _i32, _f64, _f64, _f64,
                                         _f64, _vp, _vp]),
        "gd_tm_compose": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _i32, _i32, _f64, _f64, _vp, _vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def lib() -> C.CDLL:
    """The loaded library; raises if ``libgd_poisson.so`` has not been built."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise GDError(
                        f"{LIB_PATH} is missing: build it with "
                        "`python -m gradient_domain_b200.build` (there is no CPU fallback)")
                handle = C.CDLL(LIB_PATH)
                _declare(handle)
                _lib = handle
    return _lib


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().gd_last_error().decode(errors="replace")
        raise GDError(f"{what} failed ({rc}): {msg}")


def device() -> torch.device:
    """The CUDA device used by the solvers; raises when no GPU is visible."""
    if not torch.cuda.is_available():
        raise GDError("gradient_domain_b200 needs a CUDA device (B200); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def ptr(t: torch.Tensor) -> int:
    return int(t.data_ptr())
