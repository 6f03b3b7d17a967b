"""GPU parity of the benchmark configurations' own generators against the oracle.

* Compositing (the 2048 x 2048 x 3 star-polygon case at a reduced 512 x 512
  canvas): seamless_clone(domain="mask") at a true relative residual of 1e-8
  against the reference's SuperLU masked solve (poisson.py:154-244), and the
  bench's masked system solved by a plan against SuperLU on the same system.
* The uneven batch (one plan holding Neumann integrations and masked
  composites of different sizes and channel counts): every instance against
  its own oracle, the DCT Neumann solve plus the mean fix (solvers.py:224-262)
  or SuperLU on the masked system.

Tolerance: 1e-6 relative L2 at a true relative residual of 1e-8, the accuracy
stated for the mixed-precision solver.
"""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

import gradient_domain_b200 as gd
from gradient_domain_b200 import workloads as W
from gradient_domain_b200.plan import Instance, PoissonPlan, SolveParams
from oracle import poisson as opoisson
from oracle import solvers as osolvers

pytestmark = pytest.mark.gpu

TOL = 1e-8
REL_L2 = 1e-6


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _splu_masked(f, unknown):
    """x with A x = f on the unknowns (A = -(the reference's masked matrix))."""
    interior, _, op = opoisson.masked_system(unknown)
    lu = spla.splu(op.tocsc())
    out = np.zeros_like(f)
    for c in range(f.shape[0]):
        out[c][interior] = lu.solve(-f[c][interior])
    return out


@pytest.fixture(scope="module")
def composite_512():
    return W.composite_case(512, seed=2)


def test_composite_config_seamless_clone_matches_splu(composite_512):
    src, tgt, mask = composite_512
    got, reports = gd.seamless_clone(src, tgt, mask, (0, 0), mode="import", domain="mask",
                                     tolerance=TOL)
    ref, _ = opoisson.seamless_clone(src, tgt, mask, (0, 0), mode="import", domain="mask")
    inner = np.zeros_like(mask)
    inner[1:-1, 1:-1] = mask[1:-1, 1:-1]
    assert len(reports) == 3
    for c, rep in enumerate(reports):
        assert rep.converged and rep.relative_residual <= TOL
        assert _rel(got[..., c][inner], ref[..., c][inner]) <= REL_L2
    # outside the unknowns the target is kept bit for bit (test_applications.py:65-74)
    np.testing.assert_array_equal(got[~inner], tgt[~inner])


def test_composite_config_plan_system_matches_splu(composite_512):
    src, tgt, mask = composite_512
    f_np, unk_np, _ = W.masked_system(src, tgt, mask)
    c, h, w = f_np.shape
    plan = PoissonPlan([Instance(h, w, "masked") for _ in range(c)],
                       SolveParams(tolerance=TOL, zero_start=True))
    unk = torch.as_tensor(unk_np.astype(np.uint8)).cuda()
    for k in range(c):
        plan.set_mask(k, unk)
    f = torch.as_tensor(f_np).cuda()
    x = torch.empty_like(f)
    res = plan.solve(list(f), list(x), scale=1.0)
    ref = _splu_masked(f_np, unk_np)
    got = x.cpu().numpy()
    for k in range(c):
        assert res[k].converged and res[k].relative_residual <= TOL
        assert _rel(got[k][unk_np], ref[k][unk_np]) <= REL_L2
        assert not got[k][~unk_np].any()


def test_batch_config_every_instance_matches_its_oracle():
    items = W.batch_instances(14, seed=3, side=(64, 320))
    insts, fs, masks, refs = [], [], [], []
    for it in items:
        c, h, w = it["f"].shape
        neu = it["boundary"] == "neumann"
        ref = (np.stack([osolvers.solve_neumann(-it["f"][k]) for k in range(c)]) if neu
               else _splu_masked(it["f"], it["unknown"]))
        for k in range(c):
            insts.append(Instance(h, w, it["boundary"], neu))
            fs.append(torch.as_tensor(np.ascontiguousarray(it["f"][k])).cuda())
            masks.append(None if neu else torch.as_tensor(it["unknown"].astype(np.uint8)).cuda())
            refs.append((ref[k], None if neu else it["unknown"]))
    assert {i.boundary for i in insts} == {"neumann", "masked"}
    assert len({(i.height, i.width) for i in insts}) > 5
    plan = PoissonPlan(insts, SolveParams(tolerance=TOL, zero_start=True))
    for k, m in enumerate(masks):
        if m is not None:
            plan.set_mask(k, m)
    xs = [torch.empty_like(t) for t in fs]
    res = plan.solve(fs, xs, scale=1.0)
    for k, (r, (ref, unk)) in enumerate(zip(res, refs)):
        got = xs[k].cpu().numpy()
        assert r.converged and r.relative_residual <= TOL, (k, r)
        if unk is None:
            assert abs(got.mean()) <= 1e-9 * np.abs(ref).max()
            assert _rel(got, ref) <= REL_L2, k
        else:
            assert _rel(got[unk], ref[unk]) <= REL_L2, k
