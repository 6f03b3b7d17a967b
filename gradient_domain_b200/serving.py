"""Continuous-batching Poisson server.

Requests arrive at any time and are admitted as device memory allows.  A
dispatcher groups waiting requests that can share kernel launches into a
batch and hands it to an idle worker; every batch runs on its own CUDA stream,
so batches admitted while others are still solving overlap on the device.

Request kinds (images in, image out, as the reference's editing calls):

* ``CompositeRequest`` - seamless cloning on the mask domain
  (poisson.py:261-348 with domain="mask"),
* ``FlattenRequest`` - texture flattening on the image rectangle
  (poisson.py:351-388),
* ``ToneMapRequest`` - gradient-domain tone mapping (hdr.py:137-185),
* ``PoissonRequest`` - a ready Poisson system A x = f (Neumann, Dirichlet
  rectangle or masked).

Field construction, right-hand side, solve and composition run on the device
for every kind; only the images cross PCIe.

Batching without a plan per shape.  Compositing, flattening and Dirichlet /
masked systems are all masked Poisson problems, so each one is padded to a
size bucket (sides on a geometric ladder, ratio 2^(1/4)) and solved as a masked
instance of that bucket: the unknowns are the request's own, everything
outside them is a zero Dirichlet value, which is exactly the request's system.
A batch fills the slots of a resident plan of its bucket (slot counts on a
short ladder; unused slots hold no unknowns and cost no iterations), so plans
are built per (bucket, slots) and reused by every later request of the
bucket, whatever its exact size.  Tone mapping solves its Neumann problem with
the exact DCT transform (as the reference's tone_map does), which needs no
hierarchy at all.  Ready Neumann systems keep exact-shape plans.

Plans live in one pool shared by the workers; a batch checks a plan out, so
concurrent batches of one bucket use different plans.  Resident plans are
charged to the memory budget next to the requests in flight, and idle plans
are evicted (least recently used first) when admission needs their memory.
The budget is a fraction of the device memory that was free when the server
started.

Results do not depend on the batch a request lands in beyond the solver
tolerance: every instance has its own scalars, reductions and stopping test.
Failures stay per request: a non-finite input ends its own request with
status "breakdown"; a request larger than the whole budget is rejected with
``AdmissionError``; a request cancelled before its batch starts is dropped.
"""

from __future__ import annotations

import ctypes as C
import math
import threading
import time
from collections import OrderedDict, deque
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

BYTES_PER_CELL = 16 + 60  # ready systems: f and x (FP64) plus plan workspace, per cell
MODES = ("import", "mixed", "average")


class AdmissionError(RuntimeError):
    """The request can never fit the server's device-memory budget."""


# ---------------------------------------------------------------------------
# size buckets

def _ladder(limit: int = 1 << 14) -> list[int]:
    sizes, k = [], 0
    while True:
        v = int(math.ceil(64 * 2 ** (k / 4) / 8.0)) * 8
        if not sizes or v > sizes[-1]:
            sizes.append(v)
        if v >= limit:
            return sizes
        k += 1


_SIDES = _ladder()
SLOTS = (1, 2, 3, 4, 6, 8, 12, 16, 24)


def bucket_side(n: int) -> int:
    """Smallest bucket side >= n (sides below 64 share the 64 bucket)."""
    for s in _SIDES:
        if s >= n:
            return s
    return int(math.ceil(n / 8.0)) * 8


def slot_count(channels: int) -> int:
    for k in SLOTS:
        if k >= channels:
            return k
    return channels


# ---------------------------------------------------------------------------
# requests

def _is_pinned(a) -> bool:
    return hasattr(a, "is_pinned") and a.is_pinned()


@dataclass
class PoissonRequest:
    """One Poisson system ``A x = f`` of ``channels`` right-hand sides.

    ``f`` has shape (h, w) or (c, h, w) in the library's sign convention
    (A positive); ``boundary`` is "neumann", "dirichlet" or "masked" (then
    ``unknown`` is the (h, w) bool mask of unknowns).  The result is x (c, h, w).
    """

    f: np.ndarray
    boundary: str = "neumann"
    unknown: np.ndarray | None = None
    tolerance: float = 1e-8
    tag: object = None

    def __post_init__(self):
        # f may be a NumPy array or a CPU torch tensor (pinned ones upload without a copy)
        if not hasattr(self.f, "is_pinned"):
            self.f = np.asarray(self.f, dtype=np.float64)
        if self.f.ndim == 2:
            self.f = self.f[None]
        if self.f.ndim != 3:
            raise ValueError("f must be (h, w) or (c, h, w)")
        if self.boundary not in ("neumann", "dirichlet", "masked"):
            raise ValueError(f"unknown boundary {self.boundary!r}")
        if self.boundary == "masked" and (self.unknown is None
                                          or tuple(self.unknown.shape) != tuple(self.f.shape[1:])):
            raise ValueError("masked requests need an unknown mask of shape (h, w)")

    @property
    def channels(self) -> int:
        return int(self.f.shape[0])

    @property
    def shape(self) -> tuple[int, int]:
        return int(self.f.shape[1]), int(self.f.shape[2])

    @property
    def cells(self) -> int:
        return int(np.prod(self.f.shape))

    @property
    def footprint(self) -> int:
        return self.cells * BYTES_PER_CELL

    @property
    def batch_key(self) -> tuple:
        h, w = self.shape
        if self.boundary == "neumann":
            return ("neumann", h, w, self.tolerance)
        return ("masked", bucket_side(h), bucket_side(w), self.tolerance)


def _placed_window(mask: np.ndarray, target_hw, offset, source_hw):
    """The unknowns of seamless_clone(domain="mask") on the target canvas (the
    placed mask without the image border, poisson.py:181-182) and their window
    (bounding box plus a one-pixel ring) as (interior, r0, r1, c0, c1)."""
    row, col = offset
    placed = np.zeros(target_hw, dtype=bool)
    placed[row:row + source_hw[0], col:col + source_hw[1]] = mask
    inner = np.zeros_like(placed)
    inner[1:-1, 1:-1] = placed[1:-1, 1:-1]
    rows = np.flatnonzero(inner.any(axis=1))
    if rows.size == 0:
        return placed, inner, None
    cols = np.flatnonzero(inner.any(axis=0))
    return placed, inner, (int(rows[0]) - 1, int(rows[-1]) + 2, int(cols[0]) - 1,
                           int(cols[-1]) + 2)


@dataclass
class CompositeRequest:
    """``seamless_clone(source, target, mask, offset, mode, domain="mask")``.

    The result is the composited target image; pixels outside the pasted
    selection stay bit-exact.  ``tolerance`` is the true relative residual
    of every channel's solve."""

    source: np.ndarray
    target: np.ndarray
    mask: np.ndarray
    offset: tuple = (0, 0)
    mode: str = "import"
    tolerance: float = 1e-8
    tag: object = None

    def __post_init__(self):
        self.source = np.asarray(self.source, dtype=np.float64)
        self.target = np.asarray(self.target, dtype=np.float64)
        self.mask = np.asarray(self.mask, dtype=bool)
        if self.mode not in MODES:
            raise ValueError(f"unknown mode {self.mode!r}")
        if self.source.ndim != self.target.ndim or self.target.ndim not in (2, 3):
            raise ValueError("source and target must both be (h, w) or (h, w, c)")
        if self.mask.shape != self.source.shape[:2]:
            raise ValueError("the mask must have the source's shape")
        row, col = self.offset
        h, w = self.source.shape[:2]
        if row < 0 or col < 0 or row + h > self.target.shape[0] or col + w > self.target.shape[1]:
            raise ValueError("the source patch does not fit the target at this offset")
        self.placed, self.interior, self.window = _placed_window(
            self.mask, self.target.shape[:2], self.offset, (h, w))

    @property
    def channels(self) -> int:
        return 1 if self.target.ndim == 2 else int(self.target.shape[2])

    @property
    def shape(self) -> tuple[int, int]:
        if self.window is None:
            return (0, 0)
        r0, r1, c0, c1 = self.window
        return r1 - r0, c1 - c0

    @property
    def cells(self) -> int:
        h, w = self.shape
        return h * w * self.channels

    @property
    def footprint(self) -> int:
        # target, placed source, result (images) plus field, divergence and window
        # copies per channel
        return int(self.target.size * 8 * 3 + self.cells * 8 * 4 + self.target.shape[0]
                   * self.target.shape[1])

    @property
    def batch_key(self) -> tuple:
        if self.window is None:
            return ("copy",)
        h, w = self.shape
        return ("masked", bucket_side(h), bucket_side(w), self.tolerance)


@dataclass
class FlattenRequest:
    """``texture_flatten(image, edges)`` on the image rectangle: gradients kept
    where ``edges`` (weights in [0, 1]) and the ring of ``image`` fixed."""

    image: np.ndarray
    edges: np.ndarray
    tolerance: float = 1e-8
    tag: object = None

    def __post_init__(self):
        self.image = np.asarray(self.image, dtype=np.float64)
        self.edges = np.asarray(self.edges, dtype=np.float64)
        if self.image.ndim not in (2, 3) or self.edges.shape != self.image.shape[:2]:
            raise ValueError("flattening needs an (h, w[, c]) image and (h, w) edge weights")

    @property
    def channels(self) -> int:
        return 1 if self.image.ndim == 2 else int(self.image.shape[2])

    @property
    def shape(self) -> tuple[int, int]:
        h, w = self.image.shape[:2]
        return max(h - 2, 0), max(w - 2, 0)

    @property
    def cells(self) -> int:
        h, w = self.shape
        return h * w * self.channels

    @property
    def footprint(self) -> int:
        return int(self.image.size * 8 * 4 + self.edges.size * 8)

    @property
    def batch_key(self) -> tuple:
        h, w = self.shape
        if h == 0 or w == 0:
            return ("copy",)
        return ("masked", bucket_side(h), bucket_side(w), self.tolerance)


@dataclass
class ToneMapRequest:
    """``tone_map(radiance, config)``: the display image of an (h, w, 3) radiance map.

    With ``return_factor`` the response's ``extra["factor"]`` holds the
    attenuation factor, as the reference returns it."""

    radiance: np.ndarray
    config: object = None
    return_factor: bool = False
    tag: object = None

    def __post_init__(self):
        self.radiance = np.asarray(self.radiance, dtype=np.float64)
        if self.radiance.ndim != 3 or self.radiance.shape[2] != 3:
            raise ValueError("tone mapping expects a three-channel radiance map")
        if self.config is None:
            from .hdr import ToneMapConfig
            self.config = ToneMapConfig()

    channels = 3

    @property
    def shape(self) -> tuple[int, int]:
        return int(self.radiance.shape[0]), int(self.radiance.shape[1])

    @property
    def cells(self) -> int:
        h, w = self.shape
        return h * w

    @property
    def footprint(self) -> int:
        h, w = self.shape
        return h * w * 150  # radiance, pyramid, field, transform buffer, image, result

    @property
    def batch_key(self) -> tuple:
        return ("tonemap",)


@dataclass
class Response:
    x: np.ndarray
    iterations: list
    status: list
    relative_residual: list
    submitted: float
    started: float
    finished: float
    extra: dict = field(default_factory=dict)

    @property
    def latency(self) -> float:
        return self.finished - self.submitted

    @property
    def converged(self) -> bool:
        return all(s == "converged" for s in self.status)


@dataclass
class _Job:
    request: object
    future: Future
    submitted: float
    started: float = 0.0
    taken: bool = False


# ---------------------------------------------------------------------------
# GPU backend

class _PooledPlan:
    """A resident plan with its own stream and the device buffers of its slots."""

    def __init__(self, torch, device, key, insts, params):
        from .autotune import resolve
        from .plan import PoissonPlan
        self.key = key
        self.stream = torch.cuda.Stream(device)
        with torch.cuda.device(device), torch.cuda.stream(self.stream):
            self.plan = PoissonPlan(insts, resolve(insts, params), stream=self.stream)
            k, h, w = len(insts), insts[0].height, insts[0].width
            self.f = torch.zeros((k, h, w), dtype=torch.float64, device=device)
            self.x = torch.zeros_like(self.f)
            self.masked = insts[0].boundary == "masked"
            self.m = (torch.zeros((k, h, w), dtype=torch.uint8, device=device) if self.masked
                      else None)
            self.rect = [None] * k  # slot mask is the rectangle (h, w) when set from one
        self.bytes = (self.plan.workspace_bytes + 2 * self.f.numel() * 8
                      + (self.m.numel() if self.masked else 0))
        self.last_used = time.perf_counter()

    def close(self):
        self.stream.synchronize()
        self.plan.close()


class PlanPool:
    """Resident plans of all workers, by key; a checked-out plan is not shared."""

    def __init__(self):
        self.lock = threading.Lock()
        self.idle: dict[tuple, list[_PooledPlan]] = {}
        self.resident = 0
        self.built = 0
        self.build_s = 0.0

    def checkout(self, key, build):
        with self.lock:
            plans = self.idle.get(key)
            if plans:
                return plans.pop()
        t0 = time.perf_counter()
        pp = build()
        with self.lock:
            self.resident += pp.bytes
            self.built += 1
            self.build_s += time.perf_counter() - t0
        return pp

    def checkin(self, pp: _PooledPlan):
        pp.last_used = time.perf_counter()
        with self.lock:
            self.idle.setdefault(pp.key, []).append(pp)

    def trim(self, nbytes: int) -> int:
        """Evict idle plans, least recently used first, until ``nbytes`` are freed."""
        freed = 0
        while freed < nbytes:
            with self.lock:
                cands = [(pp.last_used, key, i) for key, lst in self.idle.items()
                         for i, pp in enumerate(lst)]
                if not cands:
                    break
                _, key, i = min(cands)
                pp = self.idle[key].pop(i)
                if not self.idle[key]:
                    del self.idle[key]
                self.resident -= pp.bytes
            pp.close()
            freed += pp.bytes
        return freed

    def clear(self):
        self.trim(1 << 62)


class GpuBackend:
    """Runs one batch on the device: inputs up, fields and right-hand sides,
    one batched solve (or the tone-mapping pipeline), composition, results
    down, all on the stream of the batch's plan (or the worker's stream)."""

    def __init__(self, sweeps: int = 2, use_graph: bool = True, check_every: int = 2,
                 margin_bytes: int = 1 << 30, precision: str = "mixed", resident: bool = True):
        """``resident=False`` and ``precision="fp64"`` give the plain per-request
        baseline: every batch builds a plan of its requests' exact size, solves
        once and frees it."""
        import torch
        self.torch = torch
        self.sweeps = sweeps
        self.use_graph = use_graph
        self.check_every = check_every
        self.margin = margin_bytes
        self.precision = precision
        self.resident = resident
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.pool = PlanPool()
        # seconds the workers spent per stage, summed over batches: host staging and
        # launches of the inputs / fields / right-hand sides, the solve (until its
        # results are on the host), composition and copies down (until the stream
        # is idle), and whole tone-map batches
        self.stage_s = {"prepare": 0.0, "solve": 0.0, "finish": 0.0, "tonemap": 0.0}
        self._stage_lock = threading.Lock()

    def _stage(self, name: str, seconds: float) -> None:
        with self._stage_lock:
            self.stage_s[name] += seconds

    # -- memory ----------------------------------------------------------------
    def memory_budget(self, fraction: float) -> int:
        """``fraction`` of total device memory, but never more than what was free
        at start (minus a margin): memory other processes hold is not ours."""
        free, total = self.torch.cuda.mem_get_info(self.device)
        return int(max(0, min(fraction * total, free - self.margin)))

    def resident_bytes(self) -> int:
        return self.pool.resident

    def trim(self, nbytes: int) -> int:
        return self.pool.trim(nbytes)

    def plan_bytes(self, key, channels: int) -> int:
        """Device bytes of a plan this batch would build (an estimate, used for
        admission before the plan exists); 0 when an idle plan of its key waits."""
        if key[0] in ("masked", "neumann") and self.resident:
            pkey = (key[0], key[1], key[2], slot_count(channels), key[3])
            with self.pool.lock:
                if self.pool.idle.get(pkey):
                    return 0
        if key[0] == "masked":
            cells = key[1] * key[2] * slot_count(channels)
            return cells * (BYTES_PER_CELL + 1)
        if key[0] == "neumann":
            return key[1] * key[2] * slot_count(channels) * BYTES_PER_CELL
        return 0

    # -- workers ---------------------------------------------------------------
    def new_worker_state(self):
        return {"stream": self.torch.cuda.Stream(self.device), "dct": OrderedDict()}

    def _params(self, tol):
        from .plan import SolveParams
        return SolveParams(precision=self.precision, tolerance=tol, sweeps=self.sweeps,
                           use_graph=self.use_graph and self.resident,
                           check_every=self.check_every, zero_start=True)

    def _dct(self, state, h, w):
        from .solvers import DctPlan
        plans = state["dct"]
        plan = plans.pop((h, w), None)
        if plan is None:
            plan = DctPlan(h, w)
        plans[(h, w)] = plan
        while len(plans) > 4:
            plans.popitem(last=False)
        return plan

    def _up(self, a, dtype=None):
        """Host array (NumPy, any strides, or a pinned torch tensor) to the device on the
        current stream.  NumPy inputs of 1 MiB and more take one multi-threaded copy into
        a page-locked buffer from torch's caching host allocator (recycled once its DMA
        is done), then the DMA; a window cut from a larger image is read in place."""
        torch = self.torch
        if _is_pinned(a):
            return a.to(self.device, non_blocking=True)
        arr = np.asarray(a, dtype=dtype)
        if arr.nbytes < (1 << 20):
            return torch.from_numpy(np.ascontiguousarray(arr)).to(self.device)
        if arr.dtype == np.bool_:
            arr = arr.view(np.uint8)
        src = torch.from_numpy(arr) if all(st > 0 for st in arr.strides) else \
            torch.from_numpy(np.ascontiguousarray(arr))
        stage = torch.empty(tuple(arr.shape), dtype=src.dtype, pin_memory=True)
        stage.copy_(src)
        return stage.to(self.device, non_blocking=True)

    def _down(self, t):
        """Device tensor into a pinned host tensor on the current stream."""
        out = self.torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
        out.copy_(t, non_blocking=True)
        return out

    def _plan_for(self, requests):
        """(pool key, builder, channels) of the plan a batch of ``requests`` runs on."""
        key = requests[0].batch_key
        channels = sum(r.channels for r in requests)
        k = slot_count(channels)
        bh, bw = key[1], key[2]
        if not self.resident:  # the exact size of the batch's requests
            bh = max(r.shape[0] for r in requests)
            bw = max(r.shape[1] for r in requests)
            k = channels
        pkey = (key[0], bh, bw, k, key[3])

        def build():
            from .plan import Instance
            if pkey[0] == "masked":
                insts = [Instance(bh, bw, "masked") for _ in range(k)]
            else:
                insts = [Instance(bh, bw, "neumann", True) for _ in range(k)]
            return _PooledPlan(self.torch, self.device, pkey, insts, self._params(key[3]))

        return pkey, build, channels

    def solve(self, state, requests: list):
        key = requests[0].batch_key
        if key[0] == "tonemap":
            return self._tonemap(state, requests)
        if key[0] == "copy":
            return [self._trivial(r) for r in requests]
        pkey, build, channels = self._plan_for(requests)
        if not self.resident:
            pp = build()
            try:
                return self._solve_plan(pp, requests, channels)
            finally:
                pp.close()
        pp = self.pool.checkout(pkey, build)
        try:
            return self._solve_plan(pp, requests, channels)
        finally:
            self.pool.checkin(pp)

    def warm(self, state, requests: list, copies: int = 1) -> None:
        """Make ``copies`` resident plans for this batch (built, solved twice so their
        graphs are captured), so that as many concurrent batches of its key find a
        ready plan; tone-map batches just run once."""
        key = requests[0].batch_key
        if key[0] in ("tonemap", "copy") or not self.resident:
            self.solve(state, requests)
            return
        pkey, build, channels = self._plan_for(requests)
        plans = [self.pool.checkout(pkey, build) for _ in range(copies)]
        try:
            for pp in plans:
                for _ in range(2):
                    self._solve_plan(pp, requests, channels)
        finally:
            for pp in plans:
                self.pool.checkin(pp)

    def _trivial(self, r):
        img = r.target if isinstance(r, CompositeRequest) else r.image
        return (np.array(img, copy=True), [0] * r.channels, ["converged"] * r.channels,
                [0.0] * r.channels, {})

    def _tonemap(self, state, requests):
        torch = self.torch
        from .hdr import tone_map_device
        stream = state["stream"]
        outs = []
        t0 = time.perf_counter()
        with torch.cuda.device(self.device), torch.cuda.stream(stream):
            for r in requests:
                rad = self._up(r.radiance, np.float64)
                h, w = r.shape
                dct = self._dct(state, h, w) if min(h, w) >= 2 and max(h, w) <= 8192 else None
                img, factor = tone_map_device(rad, r.config, dct)
                outs.append((self._down(img), self._down(factor) if r.return_factor else None))
            stream.synchronize()
        self._stage("tonemap", time.perf_counter() - t0)
        res = []
        for img, factor in outs:
            extra = {"factor": factor.numpy()} if factor is not None else {}
            res.append((img.numpy(), [0] * 3, ["converged"] * 3, [0.0] * 3, extra))
        return res

    def _solve_plan(self, pp: _PooledPlan, requests, channels):
        torch = self.torch
        from ._lib import STATUS_NAMES
        from . import _lib
        lib, st = _lib.lib(), None
        k, bh, bw = pp.f.shape
        posts = []  # per request: a function of the solutions that gives its result
        t0 = time.perf_counter()
        with torch.cuda.device(self.device), torch.cuda.stream(pp.stream):
            st = _lib.stream_handle(pp.stream)
            slot = 0
            for r in requests:
                c = r.channels
                slots = list(range(slot, slot + c))
                slot += c
                posts.append((r, slots, self._prepare(pp, r, slots, lib, st)))
            for s in range(slot, k):  # unused slots: no unknowns
                pp.f[s].zero_()
                if pp.masked:
                    self._set_rect(pp, s, 0, 0)
            if pp.masked:
                pp.plan.prepare()
            t1 = time.perf_counter()
            results = pp.plan.solve(list(pp.f), list(pp.x), scale=1.0)
            t2 = time.perf_counter()
            outs = [post() for _, _, post in posts]
            pp.stream.synchronize()
        t3 = time.perf_counter()
        self._stage("prepare", t1 - t0)
        self._stage("solve", t2 - t1)
        self._stage("finish", t3 - t2)
        per = []
        for (r, slots, _), out in zip(posts, outs):
            per.append((out.numpy() if hasattr(out, "numpy") else out,
                        [results[s].iterations for s in slots],
                        [STATUS_NAMES.get(results[s].status, str(results[s].status))
                         for s in slots],
                        [results[s].relative_residual for s in slots], {}))
        return per

    def _set_rect(self, pp, s, h, w):
        """Slot s's unknowns are the rectangle [0, h) x [0, w) (none when empty)."""
        if pp.rect[s] == (h, w):
            return
        pp.m[s].zero_()
        if h and w:
            pp.m[s, :h, :w] = 1
        pp.plan.set_mask(s, pp.m[s])
        pp.rect[s] = (h, w)

    def _set_mask(self, pp, s, unk_dev, h, w):
        pp.m[s].zero_()
        pp.m[s, :h, :w] = unk_dev
        pp.plan.set_mask(s, pp.m[s])
        pp.rect[s] = None

    def _prepare(self, pp, r, slots, lib, st):
        """Upload request r, fill its slots' right-hand sides (and masks); return the
        function that turns the solutions into its result (on the plan's stream)."""
        torch = self.torch
        from . import _lib
        if isinstance(r, PoissonRequest):
            h, w = r.shape
            unk = self._up(r.unknown, np.uint8) if r.boundary == "masked" else None
            full = (h, w) == tuple(pp.f.shape[1:])
            for q, s in enumerate(slots):
                src = r.f[q]
                if full and _is_pinned(src):  # straight into the slot
                    pp.f[s].copy_(src, non_blocking=True)
                else:
                    if not full:
                        pp.f[s].zero_()
                    pp.f[s, :h, :w].copy_(self._up(src, np.float64), non_blocking=True)
                if r.boundary == "masked":
                    self._set_mask(pp, s, unk, h, w)
                elif r.boundary == "dirichlet":
                    self._set_rect(pp, s, h, w)
            return lambda: self._down(pp.x[slots[0]:slots[-1] + 1, :h, :w])
        if isinstance(r, FlattenRequest):
            return self._prepare_flatten(pp, r, slots, lib, st)
        return self._prepare_composite(pp, r, slots, lib, st)

    def _images(self, img):
        t = self._up(img[..., None] if img.ndim == 2 else img, np.float64)
        return t

    def _prepare_flatten(self, pp, r, slots, lib, st):
        torch = self.torch
        from . import _lib
        img = self._images(r.image)  # (H, W, C) on the device
        H, W, Cn = img.shape
        wts = self._up(r.edges, np.float64)
        div = torch.empty((H, W), dtype=torch.float64, device=self.device)
        bnd = torch.empty((H, W), dtype=torch.float64, device=self.device)
        f = torch.empty((H - 2, W - 2), dtype=torch.float64, device=self.device)
        for q, s in enumerate(slots):
            d = _lib.FieldDesc(_lib.GD_FIELD_WEIGHTED, H, W, Cn, q, 0, _lib.ptr(img), None, None,
                               _lib.ptr(wts), 0.0, 0.0, 0.0)
            _lib.check(lib.gd_guidance_divergence(_lib.ptr(div), C.byref(d), 0, 0, H, W, st),
                       "gd_guidance_divergence")
            bnd.copy_(img[:, :, q])
            # f = -fold(div) so that the plan solves A x = f with scale 1 (A = -laplacian)
            _lib.check(lib.gd_fold_dirichlet(_lib.ptr(f), _lib.ptr(div), _lib.ptr(bnd), H, W,
                                             -1.0, st), "gd_fold_dirichlet")
            pp.f[s].zero_()
            pp.f[s, :H - 2, :W - 2].copy_(f)
            self._set_rect(pp, s, H - 2, W - 2)

        def post():
            out = img.clone()
            out[1:-1, 1:-1, :] = pp.x[slots[0]:slots[-1] + 1, :H - 2, :W - 2].permute(1, 2, 0)
            return self._down(out[..., 0] if r.image.ndim == 2 else out)

        return post

    def _prepare_composite(self, pp, r, slots, lib, st):
        torch = self.torch
        from . import _lib
        from .poisson import _CLONE_KINDS
        tgt = self._images(r.target)  # (H, W, C)
        H, W, Cn = tgt.shape
        row, col = r.offset
        sh, sw = r.source.shape[:2]
        canvas = torch.zeros_like(tgt)
        canvas[row:row + sh, col:col + sw, :] = self._images(r.source)
        sel = self._up(r.placed, np.uint8)
        r0, r1, c0, c1 = r.window
        hh, ww = r1 - r0, c1 - c0
        unk = self._up(r.interior[r0:r1, c0:c1], np.uint8)
        div = torch.empty((hh, ww), dtype=torch.float64, device=self.device)
        win = torch.empty((hh, ww), dtype=torch.float64, device=self.device)
        f = torch.empty((hh, ww), dtype=torch.float64, device=self.device)
        kind = _CLONE_KINDS[r.mode]
        for q, s in enumerate(slots):
            d = _lib.FieldDesc(kind, H, W, Cn, q, 0, _lib.ptr(tgt), _lib.ptr(canvas),
                               _lib.ptr(sel), None, 0.0, 0.0, 0.0)
            _lib.check(lib.gd_guidance_divergence(_lib.ptr(div), C.byref(d), r0, c0, hh, ww, st),
                       "gd_guidance_divergence")
            win.copy_(tgt[r0:r1, c0:c1, q])
            _lib.check(lib.gd_masked_rhs(_lib.ptr(f), _lib.ptr(div), _lib.ptr(win),
                                         _lib.ptr(unk), hh, ww, -1.0, st), "gd_masked_rhs")
            pp.f[s].zero_()
            pp.f[s, :hh, :ww].copy_(f)
            self._set_mask(pp, s, unk, hh, ww)

        def post():
            out = tgt.clone()
            region = out[r0:r1, c0:c1, :]
            sol = pp.x[slots[0]:slots[-1] + 1, :hh, :ww].permute(1, 2, 0)
            region.copy_(torch.where(unk.bool()[..., None], sol, region))
            return self._down(out[..., 0] if r.target.ndim == 2 else out)

        return post


# ---------------------------------------------------------------------------
# server

class PoissonServer:
    """Continuous-batching server; use as a context manager or start()/stop()."""

    def __init__(self, backend=None, workers: int = 3, hbm_fraction: float = 0.8,
                 max_batch_requests: int = 16, max_batch_cells: int = 64 << 20,
                 budget_bytes: int | None = None):
        self.backend = backend if backend is not None else GpuBackend()
        self.workers = workers
        self.max_batch_requests = max_batch_requests
        self.max_batch_cells = max_batch_cells
        self.budget = (budget_bytes if budget_bytes is not None
                       else self.backend.memory_budget(hbm_fraction))
        self.in_use = 0
        self._order: deque[_Job] = deque()  # every waiting job in arrival order
        self._by_key: dict[tuple, deque[_Job]] = {}  # the same jobs by batch key
        self._waiting = 0
        self._cv = threading.Condition()
        self._idle: list[int] = list(range(workers))
        self._threads: list[threading.Thread] = []
        self._running = False
        self._states = [None] * workers
        self._work: list[list[_Job] | None] = [None] * workers
        self.batches = 0
        self.max_concurrent = 0
        self._active_batches = 0
        self.busy_s = 0.0  # worker seconds spent running batches

    # -- client side ---------------------------------------------------------
    def submit(self, request, submitted: float | None = None) -> Future:
        if request.footprint > self.budget:
            raise AdmissionError(f"request of {request.cells} cells needs "
                                 f"{request.footprint} bytes, budget {self.budget}")
        fut: Future = Future()
        job = _Job(request, fut, submitted if submitted is not None else time.perf_counter())
        with self._cv:
            if not self._running:
                raise RuntimeError("server is not running")
            self._enqueue(job)
            self._cv.notify_all()
        return fut

    def _enqueue(self, job: _Job, front: bool = False) -> None:
        job.taken = False
        q = self._by_key.setdefault(job.request.batch_key, deque())
        if front:
            q.appendleft(job)
            self._order.appendleft(job)
        else:
            q.append(job)
            self._order.append(job)
        self._waiting += 1

    @property
    def waiting(self) -> int:
        return self._waiting

    def warm(self, requests: list, batch_sizes=(1,), copies: int | None = None) -> None:
        """Prepare the plans of the batches the dispatcher will form: for every request
        and every ``b`` in ``batch_sizes``, ``copies`` (default: one per worker) resident
        plans of a batch of ``b`` copies of it, solved twice so that hierarchies,
        buffers and CUDA graphs exist before traffic arrives."""
        if self._states[0] is None:
            self._states[0] = self.backend.new_worker_state()
        copies = self.workers if copies is None else copies
        for r in requests:
            for b in batch_sizes:
                if hasattr(self.backend, "warm"):
                    self.backend.warm(self._states[0], [r] * b, copies)
                else:
                    for _ in range(2):
                        self.backend.solve(self._states[0], [r] * b)

    # -- lifecycle -----------------------------------------------------------
    def start(self):
        with self._cv:
            self._running = True
        t = threading.Thread(target=self._dispatch, name="gd-dispatch", daemon=True)
        t.start()
        self._threads.append(t)
        for wid in range(self.workers):
            w = threading.Thread(target=self._worker, args=(wid,), name=f"gd-worker{wid}",
                                 daemon=True)
            w.start()
            self._threads.append(w)
        return self

    def stop(self):
        with self._cv:
            self._running = False
            self._cv.notify_all()
        for t in self._threads:
            t.join(timeout=60)
        self._threads.clear()

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()

    # -- dispatcher ----------------------------------------------------------
    def _plan_need(self, key, channels: int) -> int:
        fn = getattr(self.backend, "plan_bytes", None)
        return fn(key, channels) if fn else 0

    def _resident(self) -> int:
        fn = getattr(self.backend, "resident_bytes", None)
        return fn() if fn else 0

    def _take_batch(self) -> list[_Job]:
        """The oldest waiting request and the later ones that share its batch key,
        as far as the batch limits and the memory budget allow.  Waiting jobs sit
        in one arrival-order queue and in a queue per key, so a batch costs time
        in its own size, however many requests wait."""
        while self._order and (self._order[0].taken or self._order[0].future.cancelled()):
            job = self._order.popleft()
            if not job.taken:  # cancelled while waiting
                job.taken = True
                self._waiting -= 1
        if not self._order:
            return []
        key = self._order[0].request.batch_key
        q = self._by_key[key]
        batch, cells, bytes_, channels = [], 0, 0, 0
        while q and len(batch) < self.max_batch_requests:
            job = q[0]
            if job.taken:
                q.popleft()
                continue
            if job.future.cancelled():
                q.popleft()
                job.taken = True
                self._waiting -= 1
                continue
            r = job.request
            if batch and (cells + r.cells > self.max_batch_cells
                          or (key[0] in ("masked", "neumann")
                              and slot_count(channels + r.channels) > SLOTS[-1])):
                break
            q.popleft()
            job.taken = True
            self._waiting -= 1
            batch.append(job)
            cells += r.cells
            bytes_ += r.footprint
            channels += r.channels
        if not q:
            del self._by_key[key]
        # memory: requests in flight, resident plans, this batch and a plan it may build
        need = bytes_ + self._plan_need(key, channels)
        over = self.in_use + self._resident() + need - self.budget
        if over > 0 and hasattr(self.backend, "trim"):
            self.backend.trim(over)
            over = self.in_use + self._resident() + need - self.budget
        while over > 0 and len(batch) > 1:  # shrink the batch until it fits
            job = batch.pop()
            self._requeue(job)
            bytes_ -= job.request.footprint
            channels -= job.request.channels
            need = bytes_ + self._plan_need(key, channels)
            over = self.in_use + self._resident() + need - self.budget
        if over > 0 and (self.in_use > 0 or self._active_batches > 0):
            for job in reversed(batch):  # wait for memory to come back
                self._requeue(job)
            return []
        started = []
        for job in batch:
            if job.future.set_running_or_notify_cancel():
                started.append(job)
        self.in_use += sum(j.request.footprint for j in started)
        return started

    def _requeue(self, job: _Job) -> None:
        """Put a job taken for a batch back at the front of the queues."""
        self._enqueue(job, front=True)

    def _dispatch(self):
        while True:
            with self._cv:
                while self._running and not (self._waiting and self._idle):
                    self._cv.wait(timeout=0.05)
                if not self._running and not self._waiting:
                    return
                if not self._idle:
                    continue
                batch = self._take_batch()
                if not batch:
                    self._cv.wait(timeout=0.001)
                    continue
                wid = self._idle.pop()
                self._active_batches += 1
                self.max_concurrent = max(self.max_concurrent, self._active_batches)
                self.batches += 1
                self._work[wid] = batch
                self._cv.notify_all()

    def _worker(self, wid: int):
        while True:
            with self._cv:
                while self._work[wid] is None and (self._running or self._waiting):
                    self._cv.wait(timeout=0.05)
                batch = self._work[wid]
                self._work[wid] = None
                if batch is None:
                    return
            self._run(wid, batch)

    def _run(self, wid: int, batch: list[_Job]):
        started = time.perf_counter()
        for job in batch:
            job.started = started
        try:
            if self._states[wid] is None:
                self._states[wid] = self.backend.new_worker_state()
            results = self.backend.solve(self._states[wid], [j.request for j in batch])
            finished = time.perf_counter()
            for job, res in zip(batch, results):
                x, its, st, rr = res[:4]
                extra = res[4] if len(res) > 4 else {}
                job.future.set_result(Response(x, its, st, rr, job.submitted, job.started,
                                               finished, extra))
        except Exception as exc:  # a failing batch fails its own requests only
            for job in batch:
                if not job.future.done():
                    job.future.set_exception(exc)
        finally:
            with self._cv:
                self.busy_s += time.perf_counter() - started
                self.in_use -= sum(j.request.footprint for j in batch)
                self._idle.append(wid)
                self._active_batches -= 1
                self._cv.notify_all()
