"""Continuous-batching Poisson solve server.

Requests (one Poisson system of one or more channels each) arrive at any time.
A dispatcher admits them into batches as device memory allows (a fraction of
HBM, 80 % by default) and hands each batch to an idle worker; every worker owns
a CUDA stream, so batches admitted while others are still solving run
concurrently on the device.  All channels of all requests of a batch are
instances of one plan, solved by the same kernel launches; plans (and with
them the multigrid hierarchies) are cached by instance list, so repeated
shapes reuse resident hierarchies.  Results do not depend on the batch a
request lands in: every instance has its own scalars and reductions, so a
request solved in a mix is bitwise equal to the same request solved alone.

Failures stay per request: a non-finite right-hand side ends that request with
status "breakdown" while its batch mates converge; a request larger than the
whole memory budget is rejected with ``AdmissionError``; a request cancelled
before its batch starts is dropped.
"""

from __future__ import annotations

import threading
import time
from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

BYTES_PER_CELL = 16 + 60  # f and x (FP64) + plan workspace (hierarchy, Krylov vectors)


class AdmissionError(RuntimeError):
    """The request can never fit the server's device-memory budget."""


@dataclass
class PoissonRequest:
    """One Poisson system ``A x = f`` of ``channels`` right-hand sides.

    ``f`` has shape (h, w) or (c, h, w) in the library's sign convention
    (A positive); ``boundary`` is "neumann", "dirichlet" or "masked" (then
    ``unknown`` is the (h, w) bool mask of unknowns).
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
                                          or self.unknown.shape != self.f.shape[1:]):
            raise ValueError("masked requests need an unknown mask of shape (h, w)")

    @property
    def cells(self) -> int:
        return int(np.prod(self.f.shape))

    @property
    def footprint(self) -> int:
        return self.cells * BYTES_PER_CELL


@dataclass
class Response:
    x: np.ndarray
    iterations: list
    status: list
    relative_residual: list
    submitted: float
    started: float
    finished: float

    @property
    def latency(self) -> float:
        return self.finished - self.submitted

    @property
    def converged(self) -> bool:
        return all(s == "converged" for s in self.status)


@dataclass
class _Job:
    request: PoissonRequest
    future: Future
    submitted: float
    started: float = 0.0


class _Staging:
    """A growing pinned host buffer reused by one worker for uploads and downloads."""

    def __init__(self, torch):
        self.torch = torch
        self.buf = None

    def get(self, n: int):
        if self.buf is None or self.buf.numel() < n:
            size = max(n, 2 * (self.buf.numel() if self.buf is not None else 0), 1 << 20)
            self.buf = self.torch.empty(size, dtype=self.torch.float64).pin_memory()
        return self.buf[:n]


class _CachedPlan:
    """A plan and the device buffers of its right-hand sides and solutions."""

    def __init__(self, torch, device, insts, params, stream):
        from .autotune import resolve
        from .plan import PoissonPlan
        self.plan = PoissonPlan(insts, resolve(insts, params), stream=stream)
        self.f = [torch.empty((i.height, i.width), dtype=torch.float64, device=device)
                  for i in insts]
        self.x = [torch.empty_like(t) for t in self.f]

    def close(self):
        self.plan.close()


class GpuBackend:
    """Solves one batch on a worker's CUDA stream through cached plans.

    A worker keeps its most recent plans with their device buffers (and, once
    solved, their captured CUDA graph), so a batch whose instance list was seen
    before costs only copies and kernel launches; inputs and results pass
    through one reusable pinned staging buffer per worker.
    """

    def __init__(self, sweeps: int = 2, use_graph: bool = True, check_every: int = 2,
                 cache_per_worker: int = 6):
        import torch
        self.torch = torch
        self.sweeps = sweeps
        self.use_graph = use_graph
        self.check_every = check_every
        self.cache_per_worker = cache_per_worker
        self.device = torch.device("cuda", torch.cuda.current_device())

    def memory_budget(self, fraction: float) -> int:
        free, total = self.torch.cuda.mem_get_info(self.device)
        return int(fraction * total)

    def new_worker_state(self):
        return {"stream": self.torch.cuda.Stream(self.device), "plans": {},
                "staging": _Staging(self.torch)}

    def _plan(self, state, insts, tol):
        from .plan import SolveParams
        key = (tuple(insts), tol)
        plans = state["plans"]
        cp = plans.pop(key, None)
        if cp is None:
            t0 = time.perf_counter()
            params = SolveParams(tolerance=tol, sweeps=self.sweeps, use_graph=self.use_graph,
                                 check_every=self.check_every, zero_start=True)
            cp = _CachedPlan(self.torch, self.device, insts, params, state["stream"])
            while len(plans) >= self.cache_per_worker:
                plans.pop(next(iter(plans))).close()
            state["plans_built"] = state.get("plans_built", 0) + 1
            state["plan_s"] = state.get("plan_s", 0.0) + time.perf_counter() - t0
        plans[key] = cp  # most recently used last
        return cp

    def solve(self, state, requests: list[PoissonRequest]):
        torch = self.torch
        from ._lib import STATUS_NAMES
        from .plan import Instance
        tol = min(r.tolerance for r in requests)
        insts, owners = [], []
        for q, r in enumerate(requests):
            c, h, w = r.f.shape
            for k in range(c):
                insts.append(Instance(h, w, r.boundary, r.boundary == "neumann"))
                owners.append((q, k))
        stream = state["stream"]
        with torch.cuda.device(self.device), torch.cuda.stream(stream):
            cp = self._plan(state, insts, tol)
            staged = [r for r in requests if not (hasattr(r.f, "is_pinned") and r.f.is_pinned())]
            total = sum(int(np.prod(r.f.shape)) for r in staged)
            stage = state["staging"].get(total) if total else None
            off = 0
            for i, (q, k) in enumerate(owners):
                src = requests[q].f
                if hasattr(src, "is_pinned") and src.is_pinned():
                    cp.f[i].copy_(src[k], non_blocking=True)
                else:
                    n = cp.f[i].numel()
                    view = stage[off:off + n]
                    np.copyto(view.numpy().reshape(cp.f[i].shape), np.asarray(src[k]))
                    cp.f[i].copy_(view.view(cp.f[i].shape), non_blocking=True)
                    off += n
            masks = {}
            for i, (q, k) in enumerate(owners):
                if requests[q].boundary == "masked":
                    if q not in masks:
                        um = requests[q].unknown
                        if not (hasattr(um, "is_pinned") and um.is_pinned()):
                            um = torch.from_numpy(
                                np.ascontiguousarray(um, dtype=np.uint8)).pin_memory()
                        masks[q] = um.to(self.device, dtype=torch.uint8, non_blocking=True)
                    cp.plan.set_mask(i, masks[q])
            results = cp.plan.solve(cp.f, cp.x, scale=1.0)
            # results go straight into pinned tensors from torch's caching host allocator
            outs = []
            for q, r in enumerate(requests):
                c, h, w = r.f.shape
                outs.append(torch.empty((c, h, w), dtype=torch.float64, pin_memory=True))
            for i, (q, k) in enumerate(owners):
                outs[q][k].copy_(cp.x[i], non_blocking=True)
            stream.synchronize()
        per, i = [], 0
        for q, r in enumerate(requests):
            c = r.f.shape[0]
            idx = list(range(i, i + c))
            i += c
            per.append((outs[q].numpy(), [results[j].iterations for j in idx],
                        [STATUS_NAMES.get(results[j].status, str(results[j].status)) for j in idx],
                        [results[j].relative_residual for j in idx]))
        return per


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
        self._pending: deque[_Job] = deque()
        self._cv = threading.Condition()
        self._idle: list[int] = list(range(workers))
        self._threads: list[threading.Thread] = []
        self._running = False
        self._states = [None] * workers
        self._work: list[list[_Job] | None] = [None] * workers
        self.batches = 0
        self.max_concurrent = 0
        self._active_batches = 0

    # -- client side ---------------------------------------------------------
    def submit(self, request: PoissonRequest, submitted: float | None = None) -> Future:
        if request.footprint > self.budget:
            raise AdmissionError(f"request of {request.cells} cells needs "
                                 f"{request.footprint} bytes, budget {self.budget}")
        fut: Future = Future()
        job = _Job(request, fut, submitted if submitted is not None else time.perf_counter())
        with self._cv:
            if not self._running:
                raise RuntimeError("server is not running")
            self._pending.append(job)
            self._cv.notify_all()
        return fut

    def warm(self, requests: list[PoissonRequest], batch_sizes=(1,)) -> None:
        """Solve batches of ``b`` copies of each request (for every ``b`` in
        ``batch_sizes``) on every worker, so that the plans of the batches the
        dispatcher will form (hierarchies, device buffers, CUDA graphs) and the
        host and device allocations behind them exist before traffic arrives."""
        for wid in range(self.workers):
            if self._states[wid] is None:
                self._states[wid] = self.backend.new_worker_state()
            for r in requests:
                for b in batch_sizes:
                    for _ in range(2):  # the second solve captures the plan's graph
                        self.backend.solve(self._states[wid], [r] * b)

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
    def _take_batch(self) -> list[_Job]:
        batch, cells, bytes_ = [], 0, 0
        while self._pending and len(batch) < self.max_batch_requests:
            job = self._pending[0]
            if job.future.cancelled():
                self._pending.popleft()
                continue
            need = job.request.footprint
            if batch and (cells + job.request.cells > self.max_batch_cells):
                break
            if self.in_use + bytes_ + need > self.budget:
                break
            self._pending.popleft()
            if not job.future.set_running_or_notify_cancel():
                continue
            batch.append(job)
            cells += job.request.cells
            bytes_ += need
        self.in_use += bytes_
        return batch

    def _dispatch(self):
        while True:
            with self._cv:
                while self._running and not (self._pending and self._idle):
                    self._cv.wait(timeout=0.05)
                if not self._running and not self._pending:
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
                while self._work[wid] is None and (self._running or self._pending):
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
            for job, (x, its, st, res) in zip(batch, results):
                job.future.set_result(Response(x, its, st, res, job.submitted, job.started,
                                               finished))
        except Exception as exc:  # a failing batch fails its own requests only
            for job in batch:
                if not job.future.done():
                    job.future.set_exception(exc)
        finally:
            with self._cv:
                self.in_use -= sum(j.request.footprint for j in batch)
                self._idle.append(wid)
                self._active_batches -= 1
                self._cv.notify_all()


# ---------------------------------------------------------------------------
# Serving benchmark: open-loop Poisson arrivals.

@dataclass
class LoadResult:
    rate: float
    requests: int
    p50_ms: float
    p99_ms: float
    solves_per_s: float
    mpix_per_s: float
    converged: int
    batches: int
    max_concurrent: int
    extra: dict = field(default_factory=dict)


def request_pool(per_type: int, seed: int, side=(256, 4096), pinned: bool = False):
    """Pre-generated requests of the three types (composite, flatten, tone-map).

    With ``pinned`` the right-hand sides are page-locked torch tensors, as a
    client that stages its inputs would submit them.
    """
    from . import workloads as W
    rng = np.random.default_rng(seed)
    pool = []
    if pinned:
        import torch

        def stage(req):
            req.f = torch.from_numpy(np.ascontiguousarray(req.f)).pin_memory()
            return req
    else:
        def stage(req):
            return req
    for k in range(3 * per_type):
        s = int(round(float(np.exp(rng.uniform(np.log(side[0]), np.log(side[1])))) / 8.0)) * 8
        kind = ("composite", "flatten", "tonemap")[k % 3]
        if kind == "tonemap":
            f = -W.neumann_blobs_shape((s, s), rng)
            pool.append(stage(PoissonRequest(f, "neumann")))
        elif kind == "flatten":
            f = np.stack([rng.standard_normal((s, s)) * 0.05 for _ in range(3)])
            pool.append(stage(PoissonRequest(f, "dirichlet")))
        else:
            mask = W.star_polygon_mask_shape((s, s), rng, rmin=0.15 * s, rmax=0.45 * s)
            unk = np.zeros_like(mask)
            unk[1:-1, 1:-1] = mask[1:-1, 1:-1]
            f = np.stack([np.where(unk, rng.standard_normal((s, s)), 0.0) for _ in range(3)])
            req = stage(PoissonRequest(f, "masked", unk))
            if pinned:
                req.unknown = torch.from_numpy(unk.astype(np.uint8)).pin_memory()
            pool.append(req)
    return pool


def run_load(server: PoissonServer, pool, rate: float, count: int, seed: int) -> LoadResult:
    """Open-loop arrivals at `rate` req/s; returns latency percentiles and throughput."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, count)
    picks = rng.integers(0, len(pool), count)
    b0 = server.batches
    states = [st for st in server._states if st is not None]
    built0 = sum(st.get("plans_built", 0) for st in states)
    plan0 = sum(st.get("plan_s", 0.0) for st in states)
    t0 = time.perf_counter()
    arrivals = t0 + np.cumsum(gaps)
    lat, fin, conv = [], [], []
    lock = threading.Lock()

    def consume(fut):
        # a client takes its result and lets it go, so pinned result buffers are recycled
        r = fut.result()
        with lock:
            lat.append(r.latency * 1e3)
            fin.append(r.finished)
            conv.append(r.converged)
        r.x = None

    futs = []
    for when, pick in zip(arrivals, picks):
        delay = when - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        fut = server.submit(pool[pick], submitted=float(when))
        fut.add_done_callback(consume)
        futs.append(fut)
    for f in futs:
        f.result()
    while True:
        with lock:
            if len(lat) == count:
                break
        time.sleep(0.001)
    t1 = max(fin)
    cells = sum(pool[p].cells for p in picks)
    lat_a = np.array(lat)
    states = [st for st in server._states if st is not None]
    extra = {"plans_built": sum(st.get("plans_built", 0) for st in states) - built0,
             "plan_build_s": round(sum(st.get("plan_s", 0.0) for st in states) - plan0, 4)}
    return LoadResult(rate, count, float(np.percentile(lat_a, 50)),
                      float(np.percentile(lat_a, 99)), count / (t1 - t0), cells / (t1 - t0) / 1e6,
                      int(sum(conv)), server.batches - b0, server.max_concurrent, extra)


def bench_main(args) -> None:
    """`bench.py --config serve`: p50 / p99 latency at several offered loads."""
    import json

    import torch

    from . import workloads as W
    torch.cuda.set_device(0)
    pool = request_pool(per_type=args.pool, seed=11, pinned=True)
    one_mp = [PoissonRequest(torch.from_numpy(-W.neumann_blobs_shape(
        (1024, 1024), np.random.default_rng(5 + i))[None].copy()).pin_memory(), "neumann")
        for i in range(8)]
    out = {"metric": "served p50/p99 latency", "unit": "ms", "config": {
        "workload": "open-loop Poisson arrivals, sides log-uniform 256-4096, "
                    "composite/flatten/tone-map", "pool_per_type": args.pool,
        "requests_per_rate": args.requests, "hbm_fraction": 0.8}}
    with PoissonServer(GpuBackend(sweeps=args.sweeps), workers=3) as server:
        run_load(server, pool, 50.0, 8, seed=1)  # warm-up: plans, allocator, kernels
        loads = []
        for rate in args.rates:
            r = run_load(server, pool, rate, args.requests, seed=int(rate))
            loads.append(r.__dict__)
        out["loads"] = loads
        server.warm(one_mp[:1], batch_sizes=(1, 2, 3))
        r1 = run_load(server, one_mp, 100.0, args.requests_1mp, seed=3)
        out["one_mp"] = r1.__dict__
        # the floor: one warm worker solving 1 MP requests back to back, no queue
        solo = []
        for i in range(100):
            t0 = time.perf_counter()
            server.backend.solve(server._states[0], [one_mp[i % len(one_mp)]])
            solo.append((time.perf_counter() - t0) * 1e3)
        out["one_mp_back_to_back_ms"] = {"p50": float(np.percentile(solo, 50)),
                                         "p99": float(np.percentile(solo, 99))}
    # per-request FP64 GPU solve, sequential, as the unbatched baseline
    from .plan import Instance, PoissonPlan, SolveParams
    t0 = time.perf_counter()
    n = 0
    for req in pool[: min(len(pool), 12)]:
        c, h, w = req.f.shape
        plan = PoissonPlan([Instance(h, w, req.boundary, req.boundary == "neumann")
                            for _ in range(c)], SolveParams(precision="fp64", use_graph=False))
        if req.boundary == "masked":
            m = torch.as_tensor(np.asarray(req.unknown)).to(torch.uint8).cuda()
            for k in range(c):
                plan.set_mask(k, m)
        f = [torch.as_tensor(np.ascontiguousarray(np.asarray(req.f[k]))).cuda() for k in range(c)]
        x = [torch.zeros_like(t) for t in f]
        plan.solve(f, x)
        _ = [t.cpu() for t in x]
        plan.close()
        n += 1
    out["fp64_sequential_solves_per_s"] = n / (time.perf_counter() - t0)
    print(json.dumps(out), flush=True)
