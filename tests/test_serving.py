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


@pytest.mark.gpu
def test_serving_mix_equals_alone():
    """A request solved in a concurrent mix equals the same request solved alone."""
    import torch

    from gradient_domain_b200.plan import Instance, PoissonPlan, SolveParams
    from gradient_domain_b200.serving import GpuBackend, request_pool
    torch.cuda.set_device(0)
    pool = request_pool(per_type=3, seed=21, side=(64, 400))
    with PoissonServer(GpuBackend(), workers=3) as srv:
        futs = [srv.submit(r) for r in pool]
        mixed = [f.result(timeout=300) for f in futs]
        assert srv.batches >= 1
    for req, got in zip(pool, mixed):
        c, h, w = req.f.shape
        plan = PoissonPlan([Instance(h, w, req.boundary, req.boundary == "neumann")
                            for _ in range(c)], SolveParams(tolerance=req.tolerance,
                                                            use_graph=False))
        if req.boundary == "masked":
            m = torch.from_numpy(req.unknown.astype(np.uint8)).cuda()
            for k in range(c):
                plan.set_mask(k, m)
        f = [torch.from_numpy(np.ascontiguousarray(req.f[k])).cuda() for k in range(c)]
        x = [torch.zeros_like(t) for t in f]
        res = plan.solve(f, x)
        alone = np.stack([t.cpu().numpy() for t in x])
        assert got.converged and all(r.converged for r in res)
        assert np.array_equal(alone, got.x)
