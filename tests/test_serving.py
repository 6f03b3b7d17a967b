"""The continuous-batching server: host logic on CPU (fake backend), mix equality on GPU."""

from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from gradient_domain_b200.serving import AdmissionError, PoissonRequest, PoissonServer


class FakeBackend:
    """Stands in for the GPU: x = f, with a delay; records batch sizes and memory."""

    def __init__(self, delay=0.02, fail_tag=None):
        self.delay = delay
        self.fail_tag = fail_tag
        self.batch_sizes = []
        self.lock = threading.Lock()
        self.active = 0
        self.max_active = 0

    def memory_budget(self, fraction):
        return int(fraction * (1 << 30))

    def new_worker_state(self):
        return {}

    def solve(self, state, requests):
        with self.lock:
            self.active += 1
            self.max_active = max(self.max_active, self.active)
            self.batch_sizes.append(len(requests))
        try:
            time.sleep(self.delay)
            if any(r.tag == self.fail_tag for r in requests if self.fail_tag is not None):
                raise RuntimeError("injected backend failure")
            out = []
            for r in requests:
                ok = np.isfinite(np.asarray(r.f)).all()
                out.append((np.array(r.f), [1] * len(r.f), ["converged" if ok else "breakdown"]
                            * len(r.f), [0.0] * len(r.f)))
            return out
        finally:
            with self.lock:
                self.active -= 1


def _req(n=16, tag=None, boundary="neumann"):
    return PoissonRequest(np.ones((2, n, n)), boundary, tag=tag)


def test_requests_are_batched_and_answered():
    be = FakeBackend(delay=0.05)
    with PoissonServer(be, workers=2, budget_bytes=1 << 30) as srv:
        futs = [srv.submit(_req()) for _ in range(20)]
        res = [f.result(timeout=30) for f in futs]
    assert all(r.converged and r.x.shape == (2, 16, 16) for r in res)
    assert len(be.batch_sizes) < 20 and sum(be.batch_sizes) == 20
    assert be.max_active <= 2


def test_oversized_request_is_rejected():
    with PoissonServer(FakeBackend(), workers=1, budget_bytes=1000) as srv:
        with pytest.raises(AdmissionError):
            srv.submit(_req(64))


def test_memory_budget_limits_what_runs_at_once():
    be = FakeBackend(delay=0.05)
    one = _req(32).footprint
    with PoissonServer(be, workers=4, budget_bytes=2 * one, max_batch_requests=1) as srv:
        futs = [srv.submit(_req(32)) for _ in range(8)]
        [f.result(timeout=30) for f in futs]
        assert srv.in_use == 0
    assert be.max_active <= 2


def test_cancelled_request_is_dropped():
    be = FakeBackend(delay=0.2)
    with PoissonServer(be, workers=1, budget_bytes=1 << 30, max_batch_requests=1) as srv:
        first = srv.submit(_req())
        time.sleep(0.05)
        second = srv.submit(_req())
        assert second.cancel()
        assert first.result(timeout=30).converged
    assert sum(be.batch_sizes) == 1


def test_failure_and_bad_input_stay_inside_their_request():
    be = FakeBackend(delay=0.01, fail_tag="boom")
    with PoissonServer(be, workers=1, budget_bytes=1 << 30, max_batch_requests=1) as srv:
        bad = PoissonRequest(np.full((1, 8, 8), np.nan), "neumann")
        f_bad = srv.submit(bad)
        f_boom = srv.submit(_req(tag="boom"))
        f_ok = srv.submit(_req())
        assert f_bad.result(timeout=30).status == ["breakdown"]
        with pytest.raises(RuntimeError):
            f_boom.result(timeout=30)
        assert f_ok.result(timeout=30).converged


def test_request_validation():
    with pytest.raises(ValueError):
        PoissonRequest(np.ones((4, 4)), "masked")
    with pytest.raises(ValueError):
        PoissonRequest(np.ones((4, 4)), "periodic")


def test_batches_share_one_key_and_keep_arrival_order():
    """A batch holds the oldest waiting request and later ones of its batch key only."""
    be = FakeBackend(delay=0.05)
    keys = []
    orig = be.solve

    def solve(state, requests):
        keys.append({r.batch_key for r in requests})
        return orig(state, requests)

    be.solve = solve
    with PoissonServer(be, workers=1, budget_bytes=1 << 30) as srv:
        block = srv.submit(_req(8))  # occupies the worker while the rest queue up
        time.sleep(0.01)
        futs = [srv.submit(_req(16 if k % 2 else 24)) for k in range(10)]
        [f.result(timeout=30) for f in [block] + futs]
    assert all(len(k) == 1 for k in keys)
    assert sum(be.batch_sizes) == 11 and len(be.batch_sizes) <= 4


def test_size_buckets_and_slot_ladder():
    from gradient_domain_b200.serving import SLOTS, bucket_side, slot_count
    sides = [bucket_side(n) for n in range(1, 5000)]
    assert all(b >= n for n, b in zip(range(1, 5000), sides))
    assert all(b % 8 == 0 for b in sides)
    assert all(b <= max(64, 1.2 * n) + 8 for n, b in zip(range(1, 5000), sides))
    assert len(set(sides)) < 30  # plans are per bucket, not per size
    assert [slot_count(c) for c in (1, 3, 5, 7, 9, 13)] == [1, 3, 6, 8, 12, 16]
    assert slot_count(SLOTS[-1] + 1) == SLOTS[-1] + 1


class PlanHoldingBackend(FakeBackend):
    """A fake whose batches leave a resident plan of ``plan`` bytes behind, which
    can be evicted (trim) only while no batch uses it."""

    def __init__(self, plan, **kw):
        super().__init__(**kw)
        self.plan = plan
        self.resident = 0
        self.trims = []

    def resident_bytes(self):
        return self.resident

    def plan_bytes(self, key, channels):
        return 0 if self.resident else self.plan

    def trim(self, nbytes):
        freed = min(self.resident, self.plan) if nbytes > 0 else 0
        self.resident -= freed
        self.trims.append(freed)
        return freed

    def solve(self, state, requests):
        with self.lock:
            self.resident = self.plan
        return super().solve(state, requests)


def test_admission_counts_resident_plans_and_evicts_them():
    """Resident plans hold budget: a request that fits only without them waits for
    an eviction instead of over-committing device memory."""
    one = _req(32).footprint
    be = PlanHoldingBackend(plan=3 * one, delay=0.02)
    with PoissonServer(be, workers=2, budget_bytes=4 * one + one // 2,
                       max_batch_requests=1) as srv:
        srv.submit(_req(32)).result(timeout=30)
        assert be.resident == 3 * one
        # the plan keeps 3 of 4.5 units: a second request fits (1 unit), a batch of two
        # would not, so the server evicts before admitting the second one concurrently
        futs = [srv.submit(_req(32)) for _ in range(2)]
        [f.result(timeout=30) for f in futs]
    assert be.max_active <= 2
    assert sum(be.trims) > 0


def test_request_kinds_validate_their_inputs():
    from gradient_domain_b200.serving import CompositeRequest, FlattenRequest, ToneMapRequest
    img = np.zeros((20, 30, 3))
    mask = np.zeros((10, 10), dtype=bool)
    mask[3:7, 3:7] = True
    r = CompositeRequest(np.ones((10, 10, 3)), img, mask, (5, 8))
    assert r.window == (7, 13, 10, 16) and r.channels == 3 and r.batch_key[0] == "masked"
    with pytest.raises(ValueError):
        CompositeRequest(np.ones((10, 10, 3)), img, mask, (15, 0))
    with pytest.raises(ValueError):
        CompositeRequest(np.ones((10, 10, 3)), img, mask, (0, 0), mode="blend")
    empty = CompositeRequest(np.ones((10, 10, 3)), img, np.zeros((10, 10), bool), (0, 0))
    assert empty.batch_key == ("copy",)
    assert FlattenRequest(img, np.ones((20, 30))).shape == (18, 28)
    with pytest.raises(ValueError):
        FlattenRequest(img, np.ones((20, 31)))
    with pytest.raises(ValueError):
        ToneMapRequest(np.ones((8, 8)))


@pytest.mark.gpu
def test_serving_mix_equals_alone():
    """Every request kind solved in a concurrent mix equals the same request served
    alone, within the solver tolerance, and matches the library's own entry point
    (seamless_clone / texture_flatten / tone_map / a plan of the exact shape)."""
    import torch

    import gradient_domain_b200 as gd
    from gradient_domain_b200 import loadgen
    from gradient_domain_b200.plan import Instance, PoissonPlan, SolveParams
    from gradient_domain_b200.serving import GpuBackend, PoissonRequest
    torch.cuda.set_device(0)
    cv = loadgen.Canvases(side=512, seed=5).build()
    reqs = [loadgen.build(loadgen.describe(s, 512, side=(64, 400)), cv) for s in range(12)]
    rng = np.random.default_rng(3)
    unk = np.zeros((90, 70), dtype=bool)
    unk[5:80, 9:60] = True
    reqs += [PoissonRequest(rng.standard_normal((2, 50, 60)), "neumann"),
             PoissonRequest(rng.standard_normal((1, 70, 40)), "dirichlet"),
             PoissonRequest(np.where(unk, rng.standard_normal((3, 90, 70)), 0.0), "masked", unk)]
    assert {type(r).__name__ for r in reqs} >= {"CompositeRequest", "FlattenRequest",
                                                "ToneMapRequest", "PoissonRequest"}
    with PoissonServer(GpuBackend(), workers=3) as srv:
        mixed = [f.result(timeout=300) for f in [srv.submit(r) for r in reqs]]
        alone = [srv.submit(r).result(timeout=300) for r in reqs]
        assert srv.backend.pool.built < 2 * len(reqs)
    for req, got, one in zip(reqs, mixed, alone):
        assert got.converged and one.converged, (type(req).__name__, got.status)
        scale = max(np.abs(one.x).max(), 1e-12)
        assert np.abs(got.x - one.x).max() <= 1e-6 * scale
        name = type(req).__name__
        if name == "CompositeRequest":
            ref, _ = gd.seamless_clone(req.source, req.target, req.mask, req.offset,
                                       domain="mask", tolerance=1e-8)
        elif name == "FlattenRequest":
            ref, _ = gd.texture_flatten(req.image, req.edges)
        elif name == "ToneMapRequest":
            ref, _ = gd.tone_map(req.radiance)
            np.testing.assert_array_equal(got.x, ref)  # same exact pipeline
            continue
        else:
            c, h, w = req.f.shape
            plan = PoissonPlan([Instance(h, w, req.boundary, req.boundary == "neumann")
                                for _ in range(c)], SolveParams(tolerance=1e-10))
            if req.boundary == "masked":
                m = torch.from_numpy(req.unknown.astype(np.uint8)).cuda()
                for k in range(c):
                    plan.set_mask(k, m)
            f = [torch.from_numpy(np.ascontiguousarray(req.f[k])).cuda() for k in range(c)]
            x = [torch.zeros_like(t) for t in f]
            plan.solve(f, x)
            ref = np.stack([t.cpu().numpy() for t in x])
        assert np.abs(got.x - ref).max() <= 1e-6 * max(np.abs(ref).max(), 1e-12), name


def test_async_batch_rejects_pageable_or_mismatched_buffers():
    """solve_neumann_batch_async checks its buffers on the host before any copy."""
    import torch
    from gradient_domain_b200 import solve_neumann_batch_async
    b = torch.zeros((2, 8, 8), dtype=torch.float64)
    with pytest.raises(ValueError):
        solve_neumann_batch_async(b, torch.zeros_like(b))          # not pinned
    with pytest.raises(ValueError):
        solve_neumann_batch_async(b.numpy(), torch.zeros_like(b))  # not a tensor
    with pytest.raises(ValueError):
        solve_neumann_batch_async(b[0], torch.zeros_like(b[0]))    # not a stack
