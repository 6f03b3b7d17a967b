"""Open-loop load for the Poisson server (the serving benchmark).

Each request is defined by its own seed: the seed draws its kind (composite,
flatten or tone-map, uniform), its side (log-uniform in [256, 4096], rounded
to a multiple of 8) and where its images come from.  The images are windows of
seeded base canvases made by the benchmark generators (blob images for
compositing and flattening, log-normal radiance modulated by blobs for tone
mapping), cut at seeded offsets, and every composite gets its own seeded
12-vertex star polygon (radii 0.15-0.39 of its side, centred), rasterised at
its size.  Requests are built by producer threads ahead of their arrival
time; a request whose inputs are not ready when it is due is submitted late
but keeps its scheduled arrival as its submit time, so producer delay counts
against the measured latency.
"""

from __future__ import annotations

import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import workloads as W
from .serving import CompositeRequest, FlattenRequest, PoissonRequest, ToneMapRequest

KINDS = ("composite", "flatten", "tonemap")


def star_mask(side: int, rng, vertices: int = 12, rmin: float = 0.146,
              rmax: float = 0.39) -> np.ndarray:
    """A centred star polygon (vertex angles 2 pi k / n + U(-0.2, 0.2), radii
    U(rmin, rmax) x side) rasterised at pixel centres by the even-odd rule.

    Scanline form of the rule: per row, each edge crossing adds one at the
    first pixel whose centre lies right of it, and a running sum along the
    row gives the crossings left of every centre (odd = inside)."""
    ang = 2 * np.pi * np.arange(vertices) / vertices + rng.uniform(-0.2, 0.2, vertices)
    rad = rng.uniform(rmin * side, rmax * side, vertices)
    c = side / 2.0
    vy, vx = c + rad * np.sin(ang), c + rad * np.cos(ang)
    yy = np.arange(side) + 0.5
    counts = np.zeros((side, side + 1), dtype=np.int8)
    j = vertices - 1
    for i in range(vertices):
        rows = np.flatnonzero((vy[i] > yy) != (vy[j] > yy))
        if rows.size:
            xint = (vx[j] - vx[i]) * (yy[rows] - vy[i]) / (vy[j] - vy[i]) + vx[i]
            first = np.clip(np.floor(xint - 0.5).astype(np.int64) + 1, 0, side)
            np.add.at(counts, (rows, first), 1)
        j = i
    return (np.cumsum(counts[:, :side], axis=1, dtype=np.int8) & 1).astype(bool)


@dataclass
class Canvases:
    """Base images the requests are cut from (side x side)."""

    side: int = 4096
    seed: int = 41
    hdr: np.ndarray = None       # (side, side, 3) radiance
    source: np.ndarray = None    # (side, side, 3) in [0, 1]
    target: np.ndarray = None
    texture: np.ndarray = None   # (side, side, 3) structure + fine texture
    edges: np.ndarray = None     # (side, side) weights in {0, 1}

    def build(self) -> "Canvases":
        rng = np.random.default_rng(self.seed)
        n = self.side
        scale = n / 1024.0
        rad = np.empty((n, n, 3))
        for c in range(3):
            mod = 0.05 + W.blob_image((n, n), 64, rng, sigma=(10.0 * scale, 120.0 * scale),
                                      noise=0.0)
            rad[..., c] = np.exp(2.5 * rng.standard_normal((n, n))) * mod
        self.hdr = rad
        self.source, self.target = W.blob_pair((n, n), 3, rng)
        structure, _ = W.blob_pair((n, n), 3, rng)
        yy, xx = np.mgrid[0:n, 0:n]
        fine = 0.04 * np.sin(0.9 * xx) * np.sin(0.7 * yy)
        self.texture = structure + fine[..., None]
        gy, gx = np.gradient(structure.mean(axis=2))
        mag = np.hypot(gx, gy)
        self.edges = (mag > np.quantile(mag, 0.9)).astype(np.float64)
        return self


@dataclass
class Descriptor:
    seed: int
    kind: str
    side: int
    offsets: tuple


def describe(seed: int, canvas_side: int, side=(256, 4096)) -> Descriptor:
    rng = np.random.default_rng(seed)
    kind = KINDS[int(rng.integers(0, 3))]
    s = int(round(float(np.exp(rng.uniform(np.log(side[0]), np.log(side[1])))) / 8.0)) * 8
    s = max(16, min(s, canvas_side))
    span = canvas_side - s
    offsets = tuple(int(v) for v in rng.integers(0, span + 1, 4))
    return Descriptor(seed, kind, s, offsets)


def build(d: Descriptor, cv: Canvases, tolerance: float = 1e-8):
    """The request of a descriptor: windows of the canvases and, for composites,
    the request's own star polygon."""
    s, (a, b, c, e) = d.side, d.offsets
    if d.kind == "tonemap":
        return ToneMapRequest(cv.hdr[a:a + s, b:b + s], tag=d.seed)
    if d.kind == "flatten":
        return FlattenRequest(cv.texture[a:a + s, b:b + s], cv.edges[a:a + s, b:b + s],
                              tolerance=tolerance, tag=d.seed)
    mask = star_mask(s, np.random.default_rng(d.seed + 1))
    return CompositeRequest(cv.source[a:a + s, b:b + s], cv.target[c:c + s, e:e + s], mask,
                            (0, 0), "import", tolerance=tolerance, tag=d.seed)


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


def run_load(server, make, count: int, rate: float, seed: int, lookahead: int = 256,
             producers: int = 8) -> LoadResult:
    """Open-loop Poisson arrivals at ``rate`` req/s of ``make(i)`` (i = 0..count-1).

    Latency is counted from the scheduled arrival to the moment the result is
    on the host."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, count)
    lat, fin, conv, late, errors = [], [], [], [], []
    cells = [0]
    lock = threading.Lock()
    done = threading.Event()
    pool = getattr(server.backend, "pool", None)
    built0 = pool.built if pool else 0
    build_s0 = pool.build_s if pool else 0.0
    b0 = server.batches
    busy0 = getattr(server, "busy_s", 0.0)
    stages0 = dict(getattr(server.backend, "stage_s", {}))

    def consume(fut):
        try:
            r = fut.result()
        except Exception as exc:  # a failed request still ends: counted, not waited for
            with lock:
                errors.append(repr(exc)[:200])
                if len(lat) + len(errors) == count:
                    done.set()
            return
        with lock:
            lat.append(r.latency * 1e3)
            fin.append(r.finished)
            conv.append(r.converged)
            if len(lat) + len(errors) == count:
                done.set()
        r.x = None  # a client takes its result and lets it go

    with ThreadPoolExecutor(max_workers=producers) as ex:
        ahead = [ex.submit(make, i) for i in range(min(lookahead, count))]
        t0 = time.perf_counter()
        arrivals = t0 + np.cumsum(gaps)
        for i, when in enumerate(arrivals):
            req = ahead[i].result()
            ahead[i] = None
            if i + lookahead < count:
                ahead.append(ex.submit(make, i + lookahead))
            delay = when - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            else:
                late.append(-delay * 1e3)
            cells[0] += req.cells
            fut = server.submit(req, submitted=float(when))
            fut.add_done_callback(consume)
    done.wait()
    t1 = max(fin) if fin else time.perf_counter()
    lat_a = np.array(lat) if lat else np.array([np.nan])
    extra = {"late_submissions": len(late),
             "late_p99_ms": float(np.percentile(late, 99)) if late else 0.0,
             "failed": len(errors), "first_errors": sorted(set(errors))[:3]}
    if hasattr(server, "busy_s"):
        extra["worker_busy"] = round((server.busy_s - busy0) / (server.workers * (t1 - t0)), 3)
    stages = getattr(server.backend, "stage_s", None)
    if stages:
        extra["stage_s"] = {k: round(v - stages0.get(k, 0.0), 3) for k, v in stages.items()}
    if pool:
        extra["plans_built"] = pool.built - built0
        extra["plan_build_s"] = round(pool.build_s - build_s0, 4)
        extra["resident_plans_gb"] = round(pool.resident / 1e9, 2)
    return LoadResult(rate, count, float(np.percentile(lat_a, 50)),
                      float(np.percentile(lat_a, 99)), count / (t1 - t0),
                      cells[0] / (t1 - t0) / 1e6, int(sum(conv)), server.batches - b0,
                      server.max_concurrent, extra)


def one_mp_requests(count: int = 8, side: int = 1024):
    """Ready 1 MP Neumann systems (the single-image integration case, blob gradient
    fields from seeds 5, 6, ...) as pinned host tensors, as a client that stages
    its inputs submits them."""
    import torch
    out = []
    for i in range(count):
        f = -W.neumann_blobs_shape((side, side), np.random.default_rng(5 + i))
        out.append(PoissonRequest(torch.from_numpy(f[None].copy()).pin_memory(), "neumann"))
    return out


def latency_1mp(server, requests: int = 300, rate: float = 100.0, seed: int = 3) -> LoadResult:
    """p50 / p99 of 1 MP Neumann requests at ``rate`` req/s (warm plans)."""
    pool = one_mp_requests()
    server.warm(pool[:1], batch_sizes=(1, 2, 3))
    return run_load(server, lambda i: pool[i % len(pool)], requests, rate, seed, producers=1)
