"""Autotuner of the plan's kernel geometry and sweeps, with a persistent cache.

The reference has one fixed V-cycle (multigrid.py:47-71: two sweeps before and
after the coarse correction); the B200 solver exposes the knobs that set how
its kernels tile the work, and the best values depend on the level sizes, the
number of instances in a plan and the boundary type:

* ``strip_target_warps`` - the height of the register-streaming strips: 0 (the
  default) chooses the height with the fewest waves x rows per launch, a
  positive value the tallest of 64/32/16/8 rows that still gives this many
  warps per launch;
* ``tile_cells`` - the largest coarse level run on shared-memory tiles rather
  than strips;
* ``bottom_cells`` - the largest level solved inside the one-CTA bottom kernel;
* ``sweeps`` - red-black sweeps per level before and after the correction
  (this trades time per iteration against iterations).

:func:`tune` times whole solves to tolerance on the device (CUDA events, the
graph path after warm-up) and runs a coordinate descent from the defaults over
:data:`SPACE`, keeping a change only when it gains at least ``min_gain``.  The
winner is cached under :func:`tune_key` - boundary types, level-0 size bucket
(powers of two of cells), instance-count bucket, precision and device name - in
memory and in a JSON file (``$GD_AUTOTUNE_CACHE``, default
``~/.cache/gradient_domain_b200/autotune.json``); :func:`lookup` returns the
cached parameters for a plan without timing anything, and :func:`resolve` -
which the plan cache, the pipelined batch solves and the serving workers call -
applies them to the fields a caller left unset (None).

Tuned parameters change the arithmetic (sweeps, which levels run on which
kernel kind), never the stopping rule: every candidate solve has to converge
to the requested tolerance, and one that does not is never chosen.
"""

from __future__ import annotations

import json
import math
import os
import threading
import time
from dataclasses import replace
from typing import Callable, Sequence

import numpy as np
import torch

from . import _lib
from .plan import Instance, PoissonPlan, SolveParams

# (parameter, candidate values); the first value of each is the default of SolveParams
SPACE: tuple[tuple[str, tuple[int, ...]], ...] = (
    ("sweeps", (2, 1, 3)),
    ("strip_target_warps", (0, 900, 3600)),
    ("tile_cells", (262144, 65536, 1048576)),
    ("bottom_cells", (4096, 1024, 16384)),
)

_CACHE_LOCK = threading.Lock()
_MEMORY: dict[tuple[str, str], dict] = {}


def cache_path() -> str:
    env = os.environ.get("GD_AUTOTUNE_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "gradient_domain_b200",
                        "autotune.json")


def device_name() -> str:
    return torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"


def tune_key(instances: Sequence[Instance], params: SolveParams | None = None,
             device: str | None = None) -> str:
    """Cache key: boundary types, level-0 size bucket, instance-count bucket, precision and
    the device the entry was timed on (entries of another GPU model never apply)."""
    params = params or SolveParams()
    if not instances:
        raise ValueError("no instances")
    kinds = "+".join(sorted({inst.boundary for inst in instances}))
    cells = max(inst.height * inst.width for inst in instances)
    size_bucket = int(round(math.log2(max(cells, 1))))
    count_bucket = 1 << int(math.ceil(math.log2(len(instances)))) if len(instances) > 1 else 1
    return (f"{kinds}|cells~2^{size_bucket}|n<={count_bucket}|{params.value('precision')}|"
            f"{device or device_name()}")


def _load(path: str) -> dict:
    try:
        with open(path) as fh:
            data = json.load(fh)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def _store(path: str, key: str, entry: dict) -> None:
    _MEMORY[(path, key)] = entry
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    data = _load(path)
    data[key] = entry
    tmp = f"{path}.tmp{os.getpid()}"
    with open(tmp, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _apply(params: SolveParams, choice: dict) -> SolveParams:
    over = {k: int(v) for k, v in choice.items() if k in dict(SPACE)}
    if choice.get("precision") in ("mixed", "fp64"):
        over["precision"] = choice["precision"]
    return replace(params, **over)


def lookup(instances: Sequence[Instance], params: SolveParams | None = None,
           path: str | None = None) -> SolveParams:
    """``params`` with the cached tuned values for this plan's key applied (unchanged if the
    key was never tuned)."""
    params = params or SolveParams()
    key = tune_key(instances, params)
    path = path or cache_path()
    with _CACHE_LOCK:
        if (path, key) in _MEMORY:
            entry = _MEMORY[(path, key)]
        else:  # read the file once per key; an untuned key is remembered as such
            entry = _load(path).get(key) or {}
            _MEMORY[(path, key)] = entry
    if not entry or entry.get("device", device_name()) != device_name():
        return params
    return _apply(params, entry.get("choice", {}))


def resolve(instances: Sequence[Instance], params: SolveParams | None = None,
            path: str | None = None) -> SolveParams:
    """The parameters a plan for ``instances`` is built with: the cached tuned values
    applied to the fields that ``params`` leaves unset (None); a value the caller set,
    even one equal to the default (e.g. ``sweeps=2``), is kept.  ``params`` itself if
    the key was never tuned."""
    params = params or SolveParams()
    tuned = lookup(instances, params, path)
    if tuned == params:
        return params
    over = {name: getattr(tuned, name) for name, _ in SPACE if getattr(params, name) is None}
    if params.precision is None:
        over["precision"] = tuned.precision
    return replace(params, **over)


def coordinate_descent(evaluate: Callable[[dict], float], start: dict,
                       space: Sequence[tuple[str, Sequence[int]]] = SPACE,
                       min_gain: float = 0.02, passes: int = 2) -> tuple[dict, float, list]:
    """Minimise ``evaluate`` one parameter at a time from ``start``.

    A candidate replaces the incumbent only when it is at least ``min_gain``
    (relative) faster, so timing noise does not move the result; a pass that
    changes nothing ends the search.  Every configuration is evaluated once.
    Returns (best choice, its cost, [(choice, cost), ...] in evaluation order).
    """
    seen: dict[tuple, float] = {}
    history: list = []

    def cost(choice: dict) -> float:
        k = tuple(sorted(choice.items()))
        if k not in seen:
            seen[k] = float(evaluate(dict(choice)))
            history.append((dict(choice), seen[k]))
        return seen[k]

    best = dict(start)
    best_cost = cost(best)
    for _ in range(max(1, passes)):
        changed = False
        for name, values in space:
            for v in values:
                if v == best.get(name):
                    continue
                cand = dict(best)
                cand[name] = v
                c = cost(cand)
                if c < best_cost * (1.0 - min_gain):
                    best, best_cost, changed = cand, c, True
        if not changed:
            break
    return best, best_cost, history


def _synthetic_rhs(inst: Instance, seed: int, dev) -> torch.Tensor:
    """A gradient-domain right-hand side: the five-point Laplacian (operators.py:86-107,
    edge-replicated for Neumann instances, zero outside for Dirichlet) of a seeded image of
    Gaussian blobs plus noise, so the solution is an image of the same size as its data,
    as in cloning, flattening and tone mapping.  (A right-hand side made of wide blobs
    itself has a solution ~N^2 larger, on which the FP32 Krylov vectors of the mixed
    solver lose most of their digits and convergence slows down, 43 iterations instead
    of 8 at 1024^2; such data wants precision="fp64".)"""
    rng = np.random.default_rng(seed)
    h, w = inst.height, inst.width
    yy = np.arange(h)[:, None]
    xx = np.arange(w)[None, :]
    img = 0.05 * rng.standard_normal((h, w))
    for _ in range(16):
        cy, cx = rng.uniform(0, h), rng.uniform(0, w)
        s = rng.uniform(0.02, 0.2) * max(h, w)
        img += rng.uniform(0, 1) * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s * s))
    mode = "edge" if inst.boundary == "neumann" else "constant"
    p = np.pad(img, 1, mode=mode)
    f = p[:-2, 1:-1] + p[2:, 1:-1] + p[1:-1, :-2] + p[1:-1, 2:] - 4.0 * img
    if inst.boundary == "neumann":
        f -= f.mean()
    return torch.as_tensor(f, dtype=torch.float64, device=dev)


def time_solve(instances: Sequence[Instance], params: SolveParams, rhs: list[torch.Tensor],
               masks: Sequence[torch.Tensor | None] | None = None, reps: int = 3,
               scale: float = 1.0) -> float:
    """Device milliseconds per solve (graph path, after two warm-up solves); infinity if an
    instance does not converge."""
    dev = rhs[0].device
    plan = PoissonPlan(list(instances), replace(params, zero_start=True))
    try:
        if masks is not None:
            for k, m in enumerate(masks):
                if m is not None:
                    plan.set_mask(k, m)
            plan.prepare()
        x = [torch.empty_like(f) for f in rhs]
        for _ in range(2):
            res = plan.solve(rhs, x, scale=scale)
        if not all(r.converged for r in res):
            return math.inf
        stream = torch.cuda.current_stream(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(reps):
            res = plan.solve(rhs, x, scale=scale)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if not all(r.converged for r in res):
            return math.inf
        return e0.elapsed_time(e1) / reps
    finally:
        plan.close()


def tune(instances: Sequence[Instance], params: SolveParams | None = None,
         rhs: list[torch.Tensor] | None = None,
         masks: Sequence[torch.Tensor | None] | None = None, reps: int = 3,
         min_gain: float = 0.02, path: str | None = None, force: bool = False,
         scale: float = 1.0, tune_precision: bool = False) -> SolveParams:
    """Tune the plan parameters for ``instances`` (see the module docstring) and cache them.

    ``rhs`` (FP64 device tensors, one per instance) defaults to seeded
    gradient-domain fields; masked instances need ``masks`` (uint8 device
    tensors of unknown cells).  With a cached entry and ``force`` false nothing
    is timed.  ``tune_precision``: also time the other precision with the
    winning geometry and keep it if faster - worth it with the caller's own
    right-hand sides, since data whose solution is dominated by the smoothest
    modes converges far slower with FP32 Krylov vectors.
    """
    params = params or SolveParams()
    instances = list(instances)
    path = path or cache_path()
    key = tune_key(instances, params)
    if not force:
        with _CACHE_LOCK:
            entry = _MEMORY.get((path, key)) or _load(path).get(key)
        if entry:
            return _apply(params, entry.get("choice", {}))
    if any(inst.boundary == "masked" for inst in instances) and masks is None:
        raise ValueError("masked instances need their masks to be tuned")
    dev = _lib.device()
    if rhs is None:
        rhs = [_synthetic_rhs(inst, 1000 + k, dev) for k, inst in enumerate(instances)]
    start = {name: values[0] for name, values in SPACE}
    t0 = time.perf_counter()
    best, best_ms, history = coordinate_descent(
        lambda choice: time_solve(instances, _apply(params, choice), rhs, masks, reps, scale),
        start, SPACE, min_gain)
    precision_ms = None
    if tune_precision:
        own = params.value("precision")
        other = "fp64" if own == "mixed" else "mixed"
        cand = dict(best, precision=other)
        ms = time_solve(instances, _apply(params, cand), rhs, masks, reps, scale)
        history.append((cand, ms))
        precision_ms = {own: best_ms, other: ms}
        if ms < best_ms * (1.0 - min_gain):
            best, best_ms = cand, ms
    if not math.isfinite(best_ms):
        raise _lib.GDError(f"autotune {key}: no configuration converged")
    entry = {"choice": best, "ms": best_ms, "default_ms": history[0][1],
             "trials": len(history), "seconds": time.perf_counter() - t0,
             "device": torch.cuda.get_device_name(dev), "min_gain": min_gain}
    if precision_ms is not None:
        entry["precision_ms"] = precision_ms
    with _CACHE_LOCK:
        _store(path, key, entry)
    return _apply(params, best)


def _main() -> None:
    import argparse

    ap = argparse.ArgumentParser(description="tune and cache plan parameters for a shape")
    ap.add_argument("--height", type=int, default=1024)
    ap.add_argument("--width", type=int, default=1024)
    ap.add_argument("--count", type=int, default=1, help="instances in the plan")
    ap.add_argument("--boundary", choices=["dirichlet", "neumann"], default="neumann")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--tolerance", type=float, default=1e-8)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    insts = [Instance(args.height, args.width, args.boundary, args.boundary == "neumann")
             for _ in range(args.count)]
    params = SolveParams(precision=args.precision, tolerance=args.tolerance)
    tuned = tune(insts, params, reps=args.reps, force=args.force)
    key = tune_key(insts, params)
    entry = _load(cache_path()).get(key, {})
    print(json.dumps({"key": key, "tuned": {k: getattr(tuned, k) for k, _ in SPACE},
                      "ms": entry.get("ms"), "default_ms": entry.get("default_ms"),
                      "trials": entry.get("trials"), "cache": cache_path()}))


if __name__ == "__main__":
    _main()
