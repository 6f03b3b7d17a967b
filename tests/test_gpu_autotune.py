"""The autotuner on the device: tuned plans still solve to tolerance and match the oracle."""

from __future__ import annotations

import json

import numpy as np
import pytest
import torch

from gradient_domain_b200 import _lib, autotune
from gradient_domain_b200.plan import Instance, PoissonPlan, SolveParams
from oracle import solvers as osolvers

pytestmark = pytest.mark.gpu


def test_tuned_plan_converges_and_matches_the_oracle(tmp_path):
    insts = [Instance(192, 256, "neumann", True), Instance(192, 256, "neumann", True)]
    params = SolveParams(tolerance=1e-8)
    path = str(tmp_path / "tune.json")
    tuned = autotune.tune(insts, params, reps=2, path=path)
    with open(path) as fh:
        entry = json.load(fh)[autotune.tune_key(insts, params)]
    assert entry["trials"] >= 5 and entry["ms"] <= entry["default_ms"]
    assert autotune.lookup(insts, params, path) == tuned
    dev = _lib.device()
    rhs = [autotune._synthetic_rhs(inst, 7 + k, dev) for k, inst in enumerate(insts)]
    plan = PoissonPlan(insts, tuned)
    x = [torch.zeros_like(f) for f in rhs]
    for _ in range(2):  # the direct-launch solve and the graph solve, both from x = 0
        for t in x:
            t.zero_()
        res = plan.solve(rhs, x, scale=-1.0)
        assert all(r.converged and r.relative_residual <= 1e-8 for r in res)
    plan.close()
    for f, u in zip(rhs, x):
        ref = osolvers.solve_neumann(f.cpu().numpy())
        got = u.cpu().numpy()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-6


def test_precision_is_tuned_on_data_that_needs_fp64(tmp_path):
    """A right-hand side made of wide blobs has a solution ~N^2 larger than its data: FP32
    Krylov vectors lose most digits there, and the tuner picks FP64 on such data."""
    n = 512
    dev = _lib.device()
    rng = np.random.default_rng(3)
    yy, xx = np.arange(n)[:, None], np.arange(n)[None, :]
    f = np.zeros((n, n))
    for _ in range(8):
        cy, cx, s = rng.uniform(0, n), rng.uniform(0, n), rng.uniform(0.05, 0.3) * n
        f += rng.uniform(-1, 1) * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s * s))
    rhs = [torch.as_tensor(f - f.mean(), device=dev)]
    insts = [Instance(n, n, "neumann", True)]
    path = str(tmp_path / "t.json")
    tuned = autotune.tune(insts, SolveParams(), rhs=rhs, reps=2, path=path, scale=-1.0,
                          tune_precision=True)
    # the data is of the kind that needs FP64: the mixed solver takes more iterations
    its = {}
    for prec in ("mixed", "fp64"):
        plan = PoissonPlan(insts, SolveParams(precision=prec, zero_start=True))
        x = [torch.empty_like(rhs[0])]
        (res,) = plan.solve(rhs, x, scale=-1.0)
        assert res.converged
        its[prec] = res.iterations
        plan.close()
    assert its["mixed"] > its["fp64"]
    # and the tuner's choice follows its own timings: the other precision only when it
    # was faster by the minimum gain
    with open(path) as fh:
        entry = json.load(fh)[autotune.tune_key(insts, SolveParams())]
    t = entry["precision_ms"]
    want = "fp64" if t["fp64"] < t["mixed"] * (1.0 - entry["min_gain"]) else "mixed"
    assert tuned.value("precision") == want
