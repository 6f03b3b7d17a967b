"""Batched solve plans: multigrid hierarchies resident on the device.

A :class:`PoissonPlan` owns one ``gd_plan`` of the C library plus its device
workspace (a torch tensor), for a fixed list of instances (grid shape and
boundary type).  Building one lays out every level of every instance and the
tile lists of all kernels; solving then costs only kernel launches.  Plans are
cached by their instance list (:func:`cached_plan`), which is what keeps the
hierarchies of repeated shapes resident across calls and across served
requests.
"""

from __future__ import annotations

import ctypes as C
import threading
from collections import OrderedDict
from dataclasses import dataclass, replace

import numpy as np
import torch

from . import _lib
from ._lib import GD_DIRICHLET, GD_FP64, GD_MASKED, GD_MIXED, GD_NEUMANN  # noqa: F401

BOUNDARIES = {"dirichlet": GD_DIRICHLET, "neumann": GD_NEUMANN, "masked": GD_MASKED}


# values of the SolveParams fields that None leaves to the library (or to the autotuner's
# cached choice for the plan's shape class, see autotune.resolve)
DEFAULTS = {"precision": "mixed", "sweeps": 2, "strip_target_warps": 0, "bottom_cells": 0,
            "tile_cells": 0}


@dataclass(frozen=True)
class SolveParams:
    """Knobs of the B200 MGPCG; the defaults follow solvers.py:171-177.

    Fields that are None take the library default (``DEFAULTS``) or, where a
    plan is built through ``autotune.resolve``, the tuned value of the plan's
    shape class; a value the caller sets, even one equal to the default, is
    always kept."""

    precision: str | None = None  # "mixed" (FP32 V-cycle, FP64 refinement) or "fp64"
    sweeps: int | None = None     # RB-GS sweeps before and after each coarse correction (2)
    max_iterations: int = 2000
    tolerance: float = 1e-8
    reliable_delta: float = 1e-4  # residual drop between FP64 residual refreshes
    check_every: int = 4          # host poll interval of solves on direct launches
    use_graph: bool = True        # from a plan's second solve on: one graph, device-side loop
    strip_target_warps: int | None = None  # strip height: 0 = fewest waves x rows, else warps per launch
    bottom_cells: int | None = None  # largest level solved inside the one-CTA bottom (0 = 4096)
    tile_cells: int | None = None    # largest coarse level on shared-memory tiles (0 = 262144)
    zero_start: bool = False      # start from x = 0; x is only written (need not be zeroed)
    persistent_coarse: bool = False  # small coarse levels + bottom in one persistent launch
    dependent_launch: bool = False   # kernels launched as programmatic dependents

    def value(self, name: str):
        """The field's value, with the library default in place of None."""
        v = getattr(self, name)
        return DEFAULTS[name] if v is None else v

    def concrete(self) -> "SolveParams":
        return replace(self, **{k: self.value(k) for k in DEFAULTS})

    def c_params(self) -> _lib.Params:
        p = self.concrete()
        return _lib.Params(GD_FP64 if p.precision == "fp64" else GD_MIXED, int(p.sweeps),
                           int(p.sweeps), int(p.max_iterations), float(p.tolerance),
                           float(p.reliable_delta), int(p.check_every),
                           1 if p.use_graph else 0, int(p.strip_target_warps),
                           int(p.bottom_cells), int(p.tile_cells),
                           1 if p.zero_start else 0, 1 if p.persistent_coarse else 0,
                           1 if p.dependent_launch else 0)


@dataclass(frozen=True)
class Instance:
    """One unknown grid: ``height x width`` cells with a boundary type."""

    height: int
    width: int
    boundary: str = "dirichlet"
    zero_mean: bool = False


@dataclass
class InstanceResult:
    iterations: int
    status: int
    relative_residual: float
    initial_norm: float
    refreshes: int = 0  # FP64 residual refreshes after the initial residual

    @property
    def converged(self) -> bool:
        return self.status == _lib.GD_CONVERGED


class PoissonPlan:
    """Hierarchies and workspace for a batch of instances on the current GPU."""

    def __init__(self, instances: list[Instance], params: SolveParams | None = None,
                 stream: torch.cuda.Stream | None = None):
        self.instances = list(instances)
        self.params = params or SolveParams()
        self.device = _lib.device()
        lib = _lib.lib()
        n = len(self.instances)
        grids = (_lib.GridDesc * n)()
        for k, inst in enumerate(self.instances):
            grids[k] = _lib.GridDesc(int(inst.height), int(inst.width),
                                     BOUNDARIES[inst.boundary], 1 if inst.zero_mean else 0)
        cp = self.params.c_params()
        handle = C.c_void_p()
        _lib.check(lib.gd_plan_create(grids, n, C.byref(cp), C.byref(handle)), "gd_plan_create")
        self._handle = handle
        nbytes = int(lib.gd_plan_workspace_bytes(handle))
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        self._stream_obj = stream if stream is not None else torch.cuda.current_stream(self.device)
        self._stream = _lib.stream_handle(stream)
        _lib.check(lib.gd_plan_bind(handle, _lib.ptr(self.workspace), nbytes, self._stream),
                   "gd_plan_bind")
        self._masked = [k for k, i in enumerate(self.instances) if i.boundary == "masked"]
        self._masks_set: set[int] = set()
        self._prepared = False
        self._reports = (_lib.Report * n)()
        self._lock = threading.Lock()
        if not self._masked:
            self.prepare()

    @property
    def workspace_bytes(self) -> int:
        return self.workspace.numel()

    def set_mask(self, index: int, unknown: torch.Tensor) -> None:
        """Unknown cells (non-zero uint8) of masked instance ``index`` (device tensor)."""
        inst = self.instances[index]
        if unknown.dtype != torch.uint8 or unknown.shape != (inst.height, inst.width):
            raise ValueError("mask must be a uint8 tensor of the instance's shape")
        unknown = unknown.contiguous()
        _lib.check(_lib.lib().gd_plan_set_mask(self._handle, index, _lib.ptr(unknown),
                                               inst.width, self._stream), "gd_plan_set_mask")
        self._masks_set.add(index)
        self._prepared = False

    def prepare(self) -> None:
        missing = set(self._masked) - self._masks_set
        if missing:
            raise RuntimeError(f"masked instances {sorted(missing)} have no mask")
        _lib.check(_lib.lib().gd_plan_prepare(self._handle, self._stream), "gd_plan_prepare")
        self._prepared = True

    def _arguments(self, rhs, x, scale):
        if not self._prepared:
            self.prepare()
        n = len(self.instances)
        if len(rhs) != n or len(x) != n:
            raise ValueError(f"expected {n} right-hand sides and solutions")
        scales = [float(scale)] * n if np.isscalar(scale) else [float(s) for s in scale]
        fp = (C.c_void_p * n)()
        xp = (C.c_void_p * n)()
        pitch = (C.c_int32 * n)()
        sc = (C.c_double * n)(*scales)
        for k, inst in enumerate(self.instances):
            for t, name in ((rhs[k], "rhs"), (x[k], "x")):
                if t.dtype != torch.float64 or t.device != self.device or t.dim() != 2:
                    raise ValueError(f"{name}[{k}] must be a 2-D float64 tensor on {self.device}")
                if tuple(t.shape) != (inst.height, inst.width) or t.stride(1) != 1:
                    raise ValueError(f"{name}[{k}] must have shape {(inst.height, inst.width)} "
                                     "with unit column stride")
            if rhs[k].stride(0) != x[k].stride(0):
                raise ValueError(f"rhs[{k}] and x[{k}] must share a row pitch")
            fp[k] = _lib.ptr(rhs[k])
            xp[k] = _lib.ptr(x[k])
            pitch[k] = x[k].stride(0)
        return fp, xp, pitch, sc

    def _results(self) -> list[InstanceResult]:
        return [InstanceResult(int(r.iterations), int(r.status), float(r.relative_residual),
                               float(r.initial_norm), int(r.refreshes)) for r in self._reports]

    def solve(self, rhs: list[torch.Tensor], x: list[torch.Tensor],
              scale: list[float] | float = 1.0) -> list[InstanceResult]:
        """Solve ``A x_i = scale_i * rhs_i`` in place in ``x`` (FP64 device tensors)."""
        fp, xp, pitch, sc = self._arguments(rhs, x, scale)
        with self._lock:
            _lib.check(_lib.lib().gd_solve(self._handle, fp, xp, pitch, sc, self._stream,
                                           self._reports), "gd_solve")
            return self._results()

    def solve_async(self, rhs: list[torch.Tensor], x: list[torch.Tensor],
                    scale: list[float] | float = 1.0) -> None:
        """Enqueue :meth:`solve` on the plan's stream; :meth:`finish` returns the results.

        From the plan's second solve on the call does not wait for the device,
        so copies and other solves can be queued behind or beside it.  ``rhs``
        and ``x`` must stay alive until :meth:`finish`.
        """
        fp, xp, pitch, sc = self._arguments(rhs, x, scale)
        with self._lock:
            _lib.check(_lib.lib().gd_solve_async(self._handle, fp, xp, pitch, sc, self._stream),
                       "gd_solve_async")

    def finish(self) -> list[InstanceResult]:
        """Wait for the solve started by :meth:`solve_async` and return its results."""
        with self._lock:
            _lib.check(_lib.lib().gd_solve_finish(self._handle, self._reports), "gd_solve_finish")
            return self._results()

    def apply_vcycle(self, index: int, r: torch.Tensor) -> torch.Tensor:
        """One V-cycle of the preconditioner on an FP64 residual (inspection hook)."""
        if not self._prepared:
            self.prepare()
        r = r.to(device=self.device, dtype=torch.float64).contiguous()
        z = torch.empty_like(r)
        _lib.check(_lib.lib().gd_plan_apply_vcycle(self._handle, index, _lib.ptr(r), _lib.ptr(z),
                                                   r.stride(0), self._stream),
                   "gd_plan_apply_vcycle")
        return z

    def set_profiling(self, enable: bool) -> None:
        """Time every kernel launch of later solves with CUDA events (no graphs)."""
        _lib.check(_lib.lib().gd_plan_set_profiling(self._handle, 1 if enable else 0),
                   "gd_plan_set_profiling")

    def kernel_times(self) -> dict[str, dict]:
        """Per kernel kind: launches, summed milliseconds and cells since profiling began."""
        n = len(_lib.KERNEL_KINDS)
        out = (_lib.KernelTime * n)()
        _lib.check(_lib.lib().gd_plan_kernel_times(self._handle, out, n), "gd_plan_kernel_times")
        return {name: {"launches": int(out[k].launches), "ms": float(out[k].milliseconds),
                       "cells": float(out[k].cells)} for k, name in enumerate(_lib.KERNEL_KINDS)}

    def level_times(self) -> dict[tuple[str, int], dict]:
        """The same totals keyed by (kind, multigrid level), launched kinds only."""
        nl = _lib.PROFILE_LEVELS
        n = len(_lib.KERNEL_KINDS) * nl
        out = (_lib.KernelTime * n)()
        _lib.check(_lib.lib().gd_plan_level_times(self._handle, out, n), "gd_plan_level_times")
        res = {}
        for k, name in enumerate(_lib.KERNEL_KINDS):
            for lvl in range(nl):
                t = out[k * nl + lvl]
                if t.launches:
                    res[(name, lvl)] = {"launches": int(t.launches), "ms": float(t.milliseconds),
                                        "cells": float(t.cells)}
        return res

    def close(self) -> None:
        if getattr(self, "_handle", None):
            # only this plan's stream can still use its workspace
            self._stream_obj.synchronize()
            _lib.lib().gd_plan_destroy(self._handle)
            self._handle = None
            self.workspace = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_CACHE: OrderedDict[tuple, PoissonPlan] = OrderedDict()
_CACHE_LOCK = threading.Lock()
CACHE_LIMIT = 32


def cached_plan(instances: tuple[Instance, ...], params: SolveParams) -> PoissonPlan:
    """A plan for this exact instance list, kept resident for reuse (LRU), built with the
    autotuner's cached parameters for its shape class where the caller left defaults."""
    from .autotune import resolve

    params = resolve(instances, params)
    key = (instances, params)
    with _CACHE_LOCK:
        plan = _CACHE.get(key)
        if plan is not None:
            _CACHE.move_to_end(key)
            return plan
    plan = PoissonPlan(list(instances), params)
    with _CACHE_LOCK:
        _CACHE[key] = plan
        while len(_CACHE) > CACHE_LIMIT:
            _, old = _CACHE.popitem(last=False)
            old.close()
    return plan


def clear_cache() -> None:
    with _CACHE_LOCK:
        while _CACHE:
            _, old = _CACHE.popitem()
            old.close()
