"""GPU parity: the CUDA path against the reference's golden vectors and the oracle.

Tolerances: reference-exact FP64 kernels match NumPy to 1e-12 relative; the
B200 MGPCG solutions match the reference solvers to 1e-6 relative L2 at a
true relative residual of 1e-8 (the target stated for this path), and to
1e-9 absolute where the drop-in runs at its direct-solver tolerance (1e-12).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import gradient_domain_b200 as gd
import mg_model as M
from gradient_domain_b200 import _lib
from gradient_domain_b200.plan import Instance, PoissonPlan, SolveParams
from oracle import operators as ops
from oracle import solvers as osolvers

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name", ["vc63", "vc47x61", "vc30x22", "vc8"])
def test_reference_vcycle_matches_golden(golden, name):
    pre, post, cs, sweeps, h = golden[f"{name}_opts"]
    opts = gd.MultigridOptions(int(pre), int(post), int(cs), int(sweeps))
    b = golden[f"{name}_b"]
    for start, key in ((np.zeros_like(b), "zero"), (golden[f"{name}_u0"], "warm")):
        got = gd.v_cycle(start, b, float(h), opts)
        ref = golden[f"{name}_{key}"]
        assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), name


def test_multigrid_solve_matches_golden_history(golden):
    u, rep = gd.solve(golden["mgsolve_b"], options=gd.MultigridOptions(tolerance=1e-10))
    assert rep.cycles == len(golden["mgsolve_hist"]) - 1
    np.testing.assert_allclose(rep.residuals, golden["mgsolve_hist"], rtol=1e-8)
    assert np.abs(u - golden["mgsolve_u"]).max() < 1e-11


@pytest.mark.parametrize("method", ["direct", "cg", "multigrid", "mgcg", "mgcg_fp64",
                                    "mgcg_port"])
def test_solve_system_matches_golden(golden, method):
    b = golden["sys_b"]
    u, rep = gd.solve_system(b, method=method, tolerance=1e-10)
    assert rep.converged and rep.relative_residual < 1e-8
    assert np.abs(u - golden["sys_direct_u"]).max() < 1e-6
    assert np.abs(u - golden["sys_exact"]).max() < 1e-6
    if method in ("cg", "multigrid"):
        assert rep.iterations == int(golden[f"sys_{method}_info"][0])
    if method == "mgcg_port":
        assert rep.iterations == int(golden["sys_mgcg_info"][0])


def test_solve_system_conventions():
    with pytest.raises(KeyError):
        gd.solve_system(np.zeros((8, 8)), method="jacobi")
    u, rep = gd.solve_system(np.zeros((16, 16)))
    assert np.all(u == 0.0) and rep.relative_residual == 0.0 and rep.converged
    b, _ = gd.manufactured_problem((33, 33), seed=10)
    u, rep = gd.solve_system(b, method="mgcg", tolerance=1e-9)
    res = float(np.linalg.norm(b - ops.laplacian(u)) / np.linalg.norm(b))
    assert res == pytest.approx(rep.relative_residual, rel=1e-6)


@pytest.mark.parametrize("key", ["neu32x40", "neu97x131", "neu64x64"])
def test_solve_neumann_matches_golden(golden, key):
    # relative to the solution's size: a rough right-hand side has a large smooth solution
    got = gd.solve_neumann(golden[f"{key}_b"])
    ref = golden[f"{key}_u"]
    assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()
    assert abs(float(got.mean())) < 1e-12


@pytest.mark.parametrize("shape", [(2, 2), (3, 5), (64, 64), (97, 130), (257, 2), (1024, 768),
                                   (7, 11), (49, 121), (1000, 1080), (2187, 6), (8192, 10),
                                   (10, 8192), (4096, 4096), (509, 1021), (128, 512),
                                   (2048, 256)])
def test_dct_neumann_matches_oracle(shape):
    """The hand-written DCT solver against the oracle's scipy DCT solve: radices 8, 4,
    2, 3, 5, 7, large primes (97, 257, 509, 1021, 13), odd lines (one unpaired row or
    column per pass) and the longest supported line (8192)."""
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    b = rng.standard_normal(shape)
    got = gd.solve_neumann(b, method="dct")
    want = osolvers.solve_neumann(b)
    assert _rel(got, want) <= 1e-12
    assert abs(got.mean()) <= 1e-12 * np.abs(got).max()


def test_dct_plans_of_different_lengths_coexist():
    """Binding a plan of short lines after one of long lines leaves the long one
    usable (the kernels' shared-memory limit is process-wide and never lowered)."""
    from gradient_domain_b200.solvers import DctPlan
    rng = np.random.default_rng(5)
    shapes = [(4096, 24), (24, 4096), (3600, 20), (40, 40), (64, 48)]
    plans = [DctPlan(*s) for s in shapes]  # long lines bound first, short ones after
    for plan, shape in zip(plans, shapes):
        b = rng.standard_normal(shape)
        bd = torch.as_tensor(b).cuda()
        got = plan.solve(bd, torch.empty_like(bd)).cpu().numpy()
        assert _rel(got, osolvers.solve_neumann(b)) <= 1e-12, shape


def test_dct_neumann_rejects_sides_beyond_its_line_limit():
    with pytest.raises(ValueError):
        gd.solve_neumann(np.zeros((8193, 4)), method="dct")
    with pytest.raises(_lib.GDError):
        from gradient_domain_b200.solvers import DctPlan
        DctPlan(4, 8193)


def test_dct_neumann_batch_matches_single():
    rng = np.random.default_rng(41)
    stack = rng.standard_normal((3, 50, 70))
    got = gd.solve_neumann_batch(stack, method="dct")
    for k in range(3):
        assert np.array_equal(got[k], gd.solve_neumann(stack[k], method="dct"))
    with pytest.raises(KeyError):
        gd.solve_neumann_batch(stack, method="fft")


@pytest.mark.parametrize("key", ["neu32x40", "neu97x131", "neu64x64"])
def test_dct_neumann_matches_golden(golden, key):
    got = gd.solve_neumann(golden[key + "_b"], method="dct")
    assert _rel(got, golden[key + "_u"]) <= 1e-12


def test_neumann_exact_on_reference_pins():
    # gradient-domain/tests/test_solvers.py:90-101
    rng = np.random.default_rng(8)
    for shape in ((64, 64), (97, 131)):
        x = rng.standard_normal(shape)
        x -= x.mean()
        assert np.abs(gd.solve_neumann(ops.neumann_laplacian(x)) - x).max() < 1e-10


@pytest.mark.parametrize("boundary,shape", [
    ("neumann", (64, 64)), ("neumann", (100, 76)), ("neumann", (257, 130)),
    ("dirichlet", (64, 64)), ("dirichlet", (129, 200)), ("dirichlet", (31, 300)),
    ("neumann", (1, 200)), ("dirichlet", (3, 5)), ("neumann", (2, 2)), ("dirichlet", (300, 1)),
])
def test_fp64_vcycle_matches_model(boundary, shape):
    rng = np.random.default_rng(sum(shape))
    r = rng.standard_normal(shape)
    plan = PoissonPlan([Instance(*shape, boundary)], SolveParams(precision="fp64", sweeps=2))
    z = plan.apply_vcycle(0, torch.as_tensor(r)).cpu().numpy()
    ref = M.vcycle(M.build_levels(shape, boundary), r, sweeps=2)
    assert _rel(z, ref) < 1e-11


@pytest.mark.parametrize("sweeps", [1, 2, 3])
def test_fp32_vcycle_matches_model(sweeps):
    rng = np.random.default_rng(sweeps)
    shape = (300, 260)
    r = rng.standard_normal(shape)
    for boundary in ("neumann", "dirichlet"):
        plan = PoissonPlan([Instance(*shape, boundary)], SolveParams(sweeps=sweeps))
        z = plan.apply_vcycle(0, torch.as_tensor(r)).cpu().numpy()
        ref = M.vcycle(M.build_levels(shape, boundary), r, sweeps=sweeps)
        assert _rel(z, ref) < 2e-5


@pytest.mark.parametrize("sweeps", [1, 2, 3])
def test_strip_height_does_not_change_the_vcycle(sweeps):
    """The strip height decides which rows near the top and bottom edges a strip
    on the interior path computes and which a strip on the general path does, so
    with interior and general arithmetic defined per cell identically, V-cycles
    with different strip heights give the same bits (two strip levels here:
    1500 x 1400 and 750 x 700), FP32 and FP64."""
    rng = np.random.default_rng(100 + sweeps)
    shape = (1500, 1400)
    r = torch.as_tensor(rng.standard_normal(shape))
    for boundary in ("neumann", "dirichlet"):
        for precision in ("mixed", "fp64"):
            outs = []
            for warps in (64, 1000, 1 << 20):  # level 0 on 64-, 16- and 8-row strips
                plan = PoissonPlan([Instance(*shape, boundary)],
                                   SolveParams(precision=precision, sweeps=sweeps,
                                               strip_target_warps=warps))
                outs.append(plan.apply_vcycle(0, r))
                plan.close()
            ref = M.vcycle(M.build_levels(shape, boundary), r.numpy(), sweeps=sweeps)
            tol = 2e-5 if precision == "mixed" else 1e-11
            assert _rel(outs[0].cpu().numpy(), ref) < tol, (boundary, precision)
            for z in outs[1:]:
                assert torch.equal(z, outs[0]), (boundary, precision)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_strip_height_does_not_change_the_solve(precision):
    """Alone, a 1500 x 1400 instance runs 8-row level-0 strips; batched with three
    2048 x 2048 instances, 64-row strips.  Its r.z partials are summed per group of
    rows whose height depends on the instance alone, so the solution and the
    iteration count are the same bits either way."""
    rng = np.random.default_rng(7)
    shapes = [(1500, 1400, "neumann")] + [(2048, 2048, "dirichlet")] * 3
    rhs = [torch.as_tensor(rng.standard_normal(s[:2])).cuda() for s in shapes]
    insts = [Instance(h, w, b, b == "neumann") for h, w, b in shapes]
    params = SolveParams(precision=precision, tolerance=1e-9, zero_start=True)
    got = []
    for members in (insts[:1], insts):
        plan = PoissonPlan(members, params)
        xs = [torch.empty_like(r) for r in rhs[:len(members)]]
        res = plan.solve(rhs[:len(members)], xs, scale=1.0)
        plan.close()
        assert all(r.converged for r in res)
        got.append((xs[0], res[0].iterations))
    assert got[0][1] == got[1][1]
    assert torch.equal(got[0][0], got[1][0])


@pytest.mark.parametrize("shape", [(1500, 1400), (301, 517), (130, 90)])
def test_full_mask_equals_dirichlet_rectangle(shape):
    """A masked instance whose mask covers the whole rectangle is the Dirichlet
    rectangle's system (walls of coefficient 1 on the finest level, 2 below), so
    its V-cycle, which runs on the masked (general) strips, gives the same bits as
    the rectangle's, which runs on the rectangle and interior strips."""
    rng = np.random.default_rng(shape[0])
    r = torch.as_tensor(rng.standard_normal(shape))
    for precision in ("mixed", "fp64"):
        rect = PoissonPlan([Instance(*shape, "dirichlet")], SolveParams(precision=precision))
        z_rect = rect.apply_vcycle(0, r)
        rect.close()
        masked = PoissonPlan([Instance(*shape, "masked")], SolveParams(precision=precision))
        masked.set_mask(0, torch.ones(shape, dtype=torch.uint8, device="cuda"))
        z_mask = masked.apply_vcycle(0, r)
        masked.close()
        assert torch.equal(z_rect, z_mask), precision


@pytest.mark.parametrize("bottom_cells", [64, 1024, 16384])
def test_bottom_sizes_give_the_same_vcycle(bottom_cells):
    """Whichever level the one-CTA bottom starts at, the V-cycle is the same."""
    rng = np.random.default_rng(bottom_cells)
    yy, xx = np.mgrid[0:300, 0:260]
    active = ((yy - 150.0) ** 2 + (xx - 130.0) ** 2 < 110.0 ** 2) & (xx % 17 != 3)
    r = rng.standard_normal((300, 260))
    for boundary in ("neumann", "dirichlet", "masked"):
        mask = active if boundary == "masked" else None
        rb = np.where(active, r, 0.0) if mask is not None else r
        for precision, tol in (("fp64", 1e-11), ("mixed", 2e-5)):
            plan = PoissonPlan([Instance(300, 260, boundary)],
                               SolveParams(precision=precision, bottom_cells=bottom_cells))
            if mask is not None:
                plan.set_mask(0, torch.as_tensor(mask.astype(np.uint8)).cuda())
            z = plan.apply_vcycle(0, torch.as_tensor(rb)).cpu().numpy()
            ref = M.vcycle(M.build_levels(rb.shape, boundary, mask), rb, sweeps=2)
            assert _rel(z, ref) < tol, (boundary, precision)


@pytest.mark.parametrize("tile_cells,sweeps", [(1, 2), (1 << 30, 1), (1 << 30, 2), (1 << 30, 3)])
def test_tile_and_strip_levels_give_the_same_vcycle(tile_cells, sweeps):
    """Coarse levels on the shared-memory tile kernels or on the strips: same V-cycle."""
    rng = np.random.default_rng(sweeps)
    yy, xx = np.mgrid[0:520, 0:300]
    active = ((yy - 260.0) ** 2 + (xx - 150.0) ** 2 < 140.0 ** 2) & (xx % 13 != 5)
    r = rng.standard_normal((520, 300))
    for boundary in ("neumann", "dirichlet", "masked"):
        mask = active if boundary == "masked" else None
        rb = np.where(active, r, 0.0) if mask is not None else r
        for precision, tol in (("fp64", 1e-11), ("mixed", 2e-5)):
            plan = PoissonPlan([Instance(520, 300, boundary)],
                               SolveParams(precision=precision, sweeps=sweeps,
                                           tile_cells=tile_cells))
            if mask is not None:
                plan.set_mask(0, torch.as_tensor(mask.astype(np.uint8)).cuda())
            z = plan.apply_vcycle(0, torch.as_tensor(rb)).cpu().numpy()
            ref = M.vcycle(M.build_levels(rb.shape, boundary, mask), rb, sweeps=sweeps)
            assert _rel(z, ref) < tol, (boundary, precision)


def test_masked_vcycle_matches_model():
    rng = np.random.default_rng(7)
    yy, xx = np.mgrid[0:300, 0:260]
    active = ((yy - 150.0) ** 2 + (xx - 130.0) ** 2 < 110.0 ** 2) & (xx % 17 != 3)
    r = np.where(active, rng.standard_normal(active.shape), 0.0)
    plan = PoissonPlan([Instance(300, 260, "masked")], SolveParams(precision="fp64", sweeps=2))
    plan.set_mask(0, torch.as_tensor(active.astype(np.uint8)).cuda())
    z = plan.apply_vcycle(0, torch.as_tensor(r)).cpu().numpy()
    ref = M.vcycle(M.build_levels(active.shape, "masked", active), r, sweeps=2)
    assert _rel(z, ref) < 1e-11


def _blob_image(shape, n, rng):
    yy, xx = np.mgrid[0:shape[0], 0:shape[1]]
    img = np.zeros(shape)
    for _ in range(n):
        cy, cx = rng.uniform(0, shape[0]), rng.uniform(0, shape[1])
        s, a = rng.uniform(10, 120), rng.uniform(0, 1)
        img += a * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s * s))
    return img + 0.05 * rng.random(shape)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_neumann_blob_1024_against_oracle(precision):
    """1024^2 Neumann integration of a blob image's gradient field, tolerance 1e-8."""
    rng = np.random.default_rng(0)
    src = _blob_image((1024, 1024), 32, rng)
    rhs = ops.divergence(*ops.gradient(src))
    oracle = osolvers.solve_neumann(rhs) + src.mean()
    plan = PoissonPlan([Instance(1024, 1024, "neumann", zero_mean=True)],
                       SolveParams(precision=precision, tolerance=1e-8))
    f = torch.as_tensor(rhs).cuda()
    x = torch.zeros_like(f)
    (res,) = plan.solve([f], [x], scale=-1.0)
    got = x.cpu().numpy() + src.mean()
    assert res.converged and res.relative_residual <= 1e-8
    assert res.iterations <= 12
    assert _rel(got, oracle) <= 1e-6
    assert _rel(got, src) <= 1e-6


def test_batch_equals_alone():
    rng = np.random.default_rng(11)
    shapes = [(64, 64, "neumann"), (200, 120, "dirichlet"), (37, 301, "neumann"),
              (130, 130, "dirichlet")]
    params = SolveParams(tolerance=1e-10)
    rhs = [torch.as_tensor(rng.standard_normal(s[:2])).cuda() for s in shapes]
    batch = PoissonPlan([Instance(*s[:2], s[2], s[2] == "neumann") for s in shapes], params)
    xb = [torch.zeros_like(r) for r in rhs]
    rb = batch.solve(rhs, xb, scale=-1.0)
    for k, s in enumerate(shapes):
        alone = PoissonPlan([Instance(*s[:2], s[2], s[2] == "neumann")], params)
        xa = torch.zeros_like(rhs[k])
        (ra,) = alone.solve([rhs[k]], [xa], scale=-1.0)
        assert rb[k].converged and ra.converged
        assert rb[k].iterations == ra.iterations
        assert torch.equal(xa, xb[k])


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_caller_buffers_of_any_alignment_and_pitch(precision):
    """Right-hand sides and solutions may be views with an odd row pitch that
    start off a 16-byte boundary (the refresh then copies element by element):
    the same bits as contiguous buffers, over repeated solves of one plan (the
    solution alternates between the caller's buffer and the plan's copy), and
    zeros where a masked instance has no unknown even from a non-zero start."""
    rng = np.random.default_rng(31)
    active = np.zeros((61, 203), bool)
    active[5:50, 7:190] = True
    active[20:30, 60:90] = False
    shapes = [(61, 203, "neumann"), (90, 131, "dirichlet"), (61, 203, "masked")]
    rhs = [rng.standard_normal(s[:2]) for s in shapes]
    start = [np.zeros(s[:2]) for s in shapes]
    start[2] = np.where(active, 0.0, 7.0)  # garbage outside the mask

    def run(offset, extra):
        plan = PoissonPlan([Instance(h, w, b, b == "neumann") for h, w, b in shapes],
                           SolveParams(precision=precision, tolerance=1e-10))
        plan.set_mask(2, torch.as_tensor(active.astype(np.uint8)).cuda())
        out = []
        for _ in range(3):
            fv, xv = [], []
            for k, (h, w, _) in enumerate(shapes):
                fb = torch.zeros((h, w + extra), dtype=torch.float64, device="cuda")
                xb = torch.zeros_like(fb)
                fb[:, offset:offset + w] = torch.as_tensor(rhs[k])
                xb[:, offset:offset + w] = torch.as_tensor(start[k])
                fv.append(fb[:, offset:offset + w])
                xv.append(xb[:, offset:offset + w])
            res = plan.solve(fv, xv, scale=-1.0)
            out.append(([t.clone() for t in xv], [(r.iterations, r.status) for r in res]))
        return out

    dense = run(0, 0)
    for offset, extra in ((1, 3), (3, 4)):
        for (xa, sa), (xb, sb) in zip(run(offset, extra), dense):
            assert sa == sb and all(s == _lib.GD_CONVERGED for _, s in sa)
            for a, b in zip(xa, xb):
                assert torch.equal(a, b)
    for xs, _ in dense:
        assert torch.all(xs[2][torch.as_tensor(~active).cuda()] == 0)
        ref = osolvers.solve_neumann(rhs[0])
        assert _rel(xs[0].cpu().numpy(), ref) < 1e-6


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_zero_start_ignores_the_initial_x(precision):
    """With zero_start the caller's x is only written: from garbage it gives the
    same bits and reports as a zero-initialised solve, including an instance
    whose right-hand side is zero (no correction is ever folded) and the graph
    solves after the first."""
    rng = np.random.default_rng(37)
    active = np.zeros((70, 90), bool)
    active[6:60, 5:80] = True
    active[20:40, 30:50] = False
    shapes = [(70, 90, "neumann"), (64, 77, "dirichlet"), (70, 90, "masked"), (40, 40, "neumann")]
    rhs = [torch.as_tensor(rng.standard_normal(s[:2])).cuda() for s in shapes]
    rhs[3] = torch.zeros((40, 40), dtype=torch.float64, device="cuda")
    runs = {}
    for zero_start in (False, True):
        plan = PoissonPlan([Instance(h, w, b, b == "neumann") for h, w, b in shapes],
                           SolveParams(precision=precision, tolerance=1e-10, zero_start=zero_start))
        plan.set_mask(2, torch.as_tensor(active.astype(np.uint8)).cuda())
        out = []
        for _ in range(3):
            xs = [torch.full_like(r, float("nan")) if zero_start else torch.zeros_like(r)
                  for r in rhs]
            res = plan.solve(rhs, xs, scale=-1.0)
            out.append(([t.clone() for t in xs],
                        [(r.iterations, r.status, r.refreshes) for r in res]))
        runs[zero_start] = out
    for (xa, sa), (xb, sb) in zip(runs[True], runs[False]):
        assert sa == sb
        for a, b in zip(xa, xb):
            assert torch.equal(a, b)
    assert torch.all(runs[True][0][0][3] == 0) and runs[True][0][1][3][0] == 0


def test_zero_and_nonfinite_rhs_are_reported_not_raised():
    plan = PoissonPlan([Instance(40, 40, "dirichlet"), Instance(40, 40, "dirichlet")],
                       SolveParams())
    f0 = torch.zeros((40, 40), dtype=torch.float64, device="cuda")
    f1 = torch.ones((40, 40), dtype=torch.float64, device="cuda")
    f1[3, 5] = float("nan")
    x0, x1 = torch.zeros_like(f0), torch.zeros_like(f1)
    r0, r1 = plan.solve([f0, f1], [x0, x1])
    assert r0.converged and r0.iterations == 0 and torch.all(x0 == 0)
    assert not r1.converged and r1.status in (_lib.GD_BREAKDOWN, _lib.GD_MAX_ITERATIONS)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_graph_solves_equal_direct_solves(precision):
    """The first solve of a plan runs on direct launches with host polls; later
    solves are one graph with a device-side while loop.  Same bits, same counts,
    and the device loop stops at the iteration cap and on zero / NaN inputs."""
    rng = np.random.default_rng(21)
    shapes = [(96, 80, "neumann"), (70, 50, "dirichlet"), (33, 129, "neumann"), (40, 40, "dirichlet")]
    rhs = [torch.as_tensor(rng.standard_normal(s[:2])).cuda() for s in shapes]
    rhs[3] = torch.zeros((40, 40), dtype=torch.float64, device="cuda")
    plan = PoissonPlan([Instance(*s[:2], s[2], s[2] == "neumann") for s in shapes],
                       SolveParams(precision=precision, tolerance=1e-10))
    runs = []
    for _ in range(3):
        xs = [torch.zeros_like(r) for r in rhs]
        res = plan.solve(rhs, xs, scale=-1.0)
        runs.append(([t.clone() for t in xs], [(r.iterations, r.status, r.refreshes) for r in res]))
    for xs, st in runs[1:]:
        assert st == runs[0][1]
        for a, b in zip(xs, runs[0][0]):
            assert torch.equal(a, b)
    assert all(r[1] == _lib.GD_CONVERGED for r in runs[0][1])
    assert all(r[2] >= 1 for r in runs[0][1][:3])  # converged through an FP64 refresh
    assert runs[0][1][3][0] == 0
    capped = PoissonPlan([Instance(96, 80, "neumann", True), Instance(40, 40, "dirichlet")],
                         SolveParams(precision=precision, tolerance=1e-14, max_iterations=2))
    bad = torch.ones((40, 40), dtype=torch.float64, device="cuda")
    bad[3, 5] = float("nan")
    for _ in range(3):
        x = [torch.zeros_like(rhs[0]), torch.zeros_like(bad)]
        r0, r1 = capped.solve([rhs[0], bad], x, scale=-1.0)
        assert r0.iterations == 2 and r0.status == _lib.GD_MAX_ITERATIONS
        assert r1.status in (_lib.GD_BREAKDOWN, _lib.GD_MAX_ITERATIONS)


def test_async_solve_and_pipelined_batch():
    rng = np.random.default_rng(23)
    f = torch.as_tensor(rng.standard_normal((70, 50))).cuda()
    plan = PoissonPlan([Instance(70, 50, "dirichlet")], SolveParams(tolerance=1e-10))
    x_sync = torch.zeros_like(f)
    (r_sync,) = plan.solve([f], [x_sync])
    for _ in range(2):  # direct launches, then the graph
        x = torch.zeros_like(f)
        plan.solve_async([f], [x])
        with pytest.raises(_lib.GDError):
            plan.solve([f], [torch.zeros_like(f)])  # one solve in flight per plan
        (r,) = plan.finish()
        assert torch.equal(x, x_sync) and r.iterations == r_sync.iterations
    with pytest.raises(_lib.GDError):
        plan.finish()
    stack = -np.stack([rng.standard_normal((64, 96)) for _ in range(3)])
    stack -= stack.mean(axis=(1, 2), keepdims=True)
    want = gd.solve_neumann_batch(stack, tolerance=1e-12)
    host_in = torch.as_tensor(stack).pin_memory()
    for _ in range(3):
        host_out = torch.full_like(host_in, 5.0).pin_memory()
        got = gd.solve_neumann_batch(host_in, tolerance=1e-12, out=host_out)
        assert got is host_out
        assert np.array_equal(host_out.numpy(), want)
        assert all(r.converged for r in gd.solve_neumann_batch.last_results)
    # several batches in flight (later uploads overlap earlier solves): each one
    # bitwise the synchronous result, also with a shape change in between
    stacks = [stack, -stack, stack[:, :48, :80].copy()]
    for k in range(2):
        stacks[2 - k] -= stacks[2 - k].mean(axis=(1, 2), keepdims=True)
    wants = [gd.solve_neumann_batch(s, tolerance=1e-12) for s in stacks]
    futs = []
    for rep in range(2):
        for s_np in stacks:
            b = torch.as_tensor(s_np).pin_memory()
            futs.append((gd.solve_neumann_batch_async(b, torch.empty_like(b).pin_memory(),
                                                      tolerance=1e-12), b))
    for k, (fut, _) in enumerate(futs):
        out = fut.result()
        assert fut.done() and fut.result() is out
        assert np.array_equal(out.numpy(), wants[k % len(stacks)])
        assert len(fut.reports) == 3 and all(r.converged for r in fut.reports)


def _device_field_div(target, kind, window, source=None, select=None, weights=None,
                      illumination=(0.0, 0.0, 0.0)):
    import ctypes as C
    t = target[..., None] if target.ndim == 2 else target
    h, w, c = t.shape
    tgt = torch.as_tensor(np.ascontiguousarray(t)).cuda()
    src = (torch.as_tensor(np.ascontiguousarray(source[..., None] if source.ndim == 2
                                                else source)).cuda()
           if source is not None else None)
    sel = torch.as_tensor(select.astype(np.uint8)).cuda() if select is not None else None
    wts = torch.as_tensor(np.ascontiguousarray(weights)).cuda() if weights is not None else None
    r0, r1, c0, c1 = window
    out = []
    for ch in range(c):
        d = _lib.FieldDesc(kind, h, w, c, ch, 0, _lib.ptr(tgt),
                           _lib.ptr(src) if src is not None else None,
                           _lib.ptr(sel) if sel is not None else None,
                           _lib.ptr(wts) if wts is not None else None, *illumination)
        div = torch.empty((r1 - r0, c1 - c0), dtype=torch.float64, device="cuda")
        _lib.check(_lib.lib().gd_guidance_divergence(_lib.ptr(div), C.byref(d), r0, c0,
                                                     r1 - r0, c1 - c0, _lib.stream_handle()),
                   "gd_guidance_divergence")
        out.append(div.cpu().numpy())
    return out


def test_device_guidance_fields_match_numpy_fields():
    """gd_guidance_divergence forms the editing fields and their divergence on the
    device: bitwise the NumPy result for cloning and weighted fields, to rounding
    for the illumination remap (its power function may differ in the last bit)."""
    from oracle import poisson as op
    rng = np.random.default_rng(31)
    target = rng.random((70, 90, 3))
    source = rng.random((40, 50, 3))
    yy, xx = np.mgrid[0:40, 0:50]
    mask = (yy - 20.0) ** 2 / 300 + (xx - 25.0) ** 2 / 500 < 1.0
    offset = (12, 21)
    window = (5, 66, 8, 85)
    win = (slice(window[0], window[1]), slice(window[2], window[3]))
    inner = (slice(1, -1), slice(1, -1))
    kinds = {"import": _lib.GD_FIELD_IMPORT, "mixed": _lib.GD_FIELD_MIXED,
             "average": _lib.GD_FIELD_AVERAGE}
    for mode, kind in kinds.items():
        field, placed, tgt = op.clone_field(source, target, mask, offset, mode)
        canvas, _ = op.place(source, mask, target.shape, offset)
        got = _device_field_div(target, kind, window, source=canvas, select=placed)
        for ch in range(3):
            want = ops.divergence(field.gx[win][..., ch], field.gy[win][..., ch])
            assert np.array_equal(got[ch][inner], want[inner]), mode
    weights = (rng.random((70, 90)) > 0.6).astype(float) * rng.random((70, 90))
    g = op.GuidanceField.of(target).scaled(weights[..., None])
    got = _device_field_div(target, _lib.GD_FIELD_WEIGHTED, window, weights=weights)
    for ch in range(3):
        want = ops.divergence(g.gx[win][..., ch], g.gy[win][..., ch])
        assert np.array_equal(got[ch][inner], want[inner])
    alpha, beta, eps = 0.2, 0.3, 1e-4
    f = op.GuidanceField.of(target)
    factor = (alpha ** beta) * np.maximum(np.sqrt(f.gx ** 2 + f.gy ** 2), eps) ** (-beta)
    g = f.scaled(factor)
    got = _device_field_div(target, _lib.GD_FIELD_ILLUMINATION, window,
                            illumination=(alpha ** beta, beta, eps))
    for ch in range(3):
        want = ops.divergence(g.gx[win][..., ch], g.gy[win][..., ch])
        assert np.abs(got[ch][inner] - want[inner]).max() <= 1e-14 * np.abs(want).max()


def test_masked_and_dirichlet_applications_match_golden(golden):
    field = gd.GuidanceField.of(golden["app_src"])
    got, reps = gd.solve_masked(field, golden["app_img"], golden["app_disc"])
    assert len(reps) == 3 and all(r.converged for r in reps)
    assert np.abs(got - golden["app_masked"]).max() < 1e-9
    outside = ~golden["app_disc"]
    assert np.array_equal(got[outside], golden["app_img"][outside])
    got, reps = gd.solve_dirichlet(field, golden["app_img"], method="mgcg", tolerance=1e-12)
    assert np.abs(got - golden["app_dirichlet"]).max() < 1e-9
    got, _ = gd.solve_dirichlet(field, golden["app_img"], method="direct")
    assert np.abs(got - golden["app_dirichlet"]).max() < 1e-9


def test_editing_entry_points_match_golden(golden):
    off = tuple(int(v) for v in golden["clone_offset"])
    for mode in ("import", "mixed", "average"):
        got, _ = gd.seamless_clone(golden["clone_source"], golden["clone_target"],
                                   golden["clone_mask"], off, mode=mode, domain="mask")
        assert np.abs(got - golden[f"clone_{mode}_mask"]).max() < 1e-9, mode
    got, _ = gd.seamless_clone(golden["clone_source"], golden["clone_target"],
                               golden["clone_mask"], off, domain="rectangle", method="direct")
    assert np.abs(got - golden["clone_import_rect"]).max() < 1e-9
    got, _ = gd.texture_flatten(golden["tex_image"], golden["tex_edges"], method="direct")
    assert np.abs(got - golden["tex_flat"]).max() < 1e-9
    got, _ = gd.illumination_change(golden["tex_image"], golden["illum_mask"], alpha=0.4,
                                    beta=0.6)
    assert np.abs(got - golden["illum"]).max() < 1e-9
    with pytest.raises(ValueError):
        gd.seamless_clone(golden["clone_source"], golden["clone_target"], golden["clone_mask"],
                          off, mode="blend")
    with pytest.raises(ValueError):
        gd.seamless_clone(golden["clone_source"], golden["clone_target"], golden["clone_mask"],
                          off, domain="triangle")


def test_tone_map_matches_golden(golden):
    mapped, factor = gd.tone_map(golden["tm_radiance"])
    np.testing.assert_allclose(factor, golden["tm_factor"], rtol=1e-12)
    assert np.abs(mapped - golden["tm_mapped"]).max() < 1e-8
    with pytest.raises(ValueError):
        gd.tone_map(np.ones((16, 16)))


@pytest.mark.parametrize("shape,levels", [((300, 257), 8), ((97, 130), 3), ((40, 33), 8)])
def test_tone_map_matches_oracle(shape, levels):
    """The device tone map (pyramid, field, Neumann solve, exposure and the exact
    radix-selected percentile) against the oracle's NumPy/DCT pipeline; the
    radiance repeats values so the percentile meets ties."""
    from oracle import hdr as oh
    rng = np.random.default_rng(sum(shape))
    rad = np.exp(2.0 * rng.standard_normal(shape + (3,)))
    rad[: shape[0] // 3] = np.round(rad[: shape[0] // 3], 1) + 0.1
    cfg = gd.ToneMapConfig(levels=levels)
    got, fgot = gd.tone_map(rad, cfg)
    want, fwant = oh.tone_map(rad, oh.ToneMapConfig(levels=levels))
    np.testing.assert_allclose(fgot, fwant, rtol=1e-12)
    assert np.abs(got - want).max() < 1e-8
    np.testing.assert_allclose(gd.attenuation_field(np.log(rad[..., 0]), cfg),
                               oh.attenuation_field(np.log(rad[..., 0]),
                                                    oh.ToneMapConfig(levels=levels)), rtol=1e-12)


def test_operators_match_golden(golden):
    gx, gy = gd.gradient(golden["op_u"])
    np.testing.assert_array_equal(gx, golden["op_gx"])
    np.testing.assert_array_equal(gy, golden["op_gy"])
    np.testing.assert_array_equal(gd.divergence(golden["op_vx"], golden["op_vy"]),
                                  golden["op_div"])
    np.testing.assert_array_equal(gd.laplacian(golden["op_u"], 0.5), golden["op_lap_h05"])
    # the reference's fold at spacing 0.5 (operators.py:139-169), on the device
    np.testing.assert_array_equal(gd.fold_boundary(np.zeros((12, 16)), golden["op_ring"], 0.5),
                                  golden["op_fold"])


def test_transfers_match_golden(golden):
    """Full-weighting restriction and bilinear prolongation of the reference
    (multigrid.py:169-181) on the device."""
    from gradient_domain_b200.multigrid import _prolong, _restrict
    np.testing.assert_allclose(_restrict(golden["tr_fine"]), golden["tr_restrict"], rtol=1e-12,
                               atol=1e-15)
    np.testing.assert_allclose(_prolong(golden["tr_coarse"], (31, 25)), golden["tr_prolong"],
                               rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("shape,channels,spacing", [((14, 18), 0, 1.0), ((14, 18), 3, 0.5),
                                                    ((3, 3), 2, 0.3), ((3, 40), 1, 2.0),
                                                    ((57, 4), 4, 0.75)])
def test_fold_boundary_on_device_matches_oracle(shape, channels, spacing):
    """Multichannel and spacing != 1 fold on the device, bitwise the reference's
    sequence of subtractions (corners take two, in the reference's order)."""
    rng = np.random.default_rng(sum(shape) + channels)
    extra = (channels,) if channels else ()
    bnd = rng.standard_normal(shape + extra)
    rhs = rng.standard_normal((shape[0] - 2, shape[1] - 2) + extra)
    got = gd.fold_boundary(rhs, bnd, spacing)
    np.testing.assert_array_equal(got, ops.fold_boundary(rhs, bnd, spacing))
    # the reference's own pins (test_operators.py:78-90): the fold completes the stencil
    full = rng.standard_normal(shape)
    folded = ops.laplacian(full[1:-1, 1:-1]) - gd.fold_boundary(np.zeros(
        (shape[0] - 2, shape[1] - 2)), full)
    np.testing.assert_allclose(folded, ops.laplacian(full)[1:-1, 1:-1], atol=1e-12)
    with pytest.raises(ValueError):
        gd.fold_boundary(rhs, bnd[:-1], spacing)


def test_bounded_wait_gives_up_and_reports():
    """A bulk-copy wait whose bytes never arrive gives up after its attempt limit,
    sets the error bit and returns; the context stays usable (a solve follows)."""
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    done = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    _lib.check(_lib.lib().gd_selftest_bounded_wait(2000, _lib.ptr(err), _lib.ptr(done),
                                                   _lib.stream_handle()),
               "gd_selftest_bounded_wait")
    torch.cuda.synchronize()
    assert err.item() == 1 and done.item() == 0
    with pytest.raises(_lib.GDError):
        _lib.check(_lib.lib().gd_selftest_bounded_wait(0, _lib.ptr(err), _lib.ptr(done),
                                                       _lib.stream_handle()),
                   "gd_selftest_bounded_wait")
    f = torch.as_tensor(np.random.default_rng(5).standard_normal((64, 64))).cuda()
    x = torch.empty_like(f)
    plan = PoissonPlan([Instance(64, 64, "neumann", True)], SolveParams(zero_start=True))
    (res,) = plan.solve([f], [x], scale=-1.0)
    assert res.converged


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_persistent_coarse_launch_equals_level_launches(precision):
    """The coarse levels and the bottom in one persistent cooperative launch give
    bitwise the results of one launch per level (the same per-tile and per-instance
    device functions run in the same order), on an uneven batch of all boundary
    types, on direct launches and on the graph of later solves."""
    rng = np.random.default_rng(17)
    shapes = [(1100, 900, "neumann"), (700, 1300, "dirichlet"), (600, 640, "masked"),
              (300, 200, "neumann"), (90, 70, "dirichlet")]
    yy, xx = np.mgrid[0:600, 0:640]
    mask = ((yy - 300.0) ** 2 + (xx - 320.0) ** 2 < 260.0 ** 2).astype(np.uint8)
    rhs = []
    for h, w, kind in shapes:
        f = rng.standard_normal((h, w))
        if kind == "masked":
            f = np.where(mask, f, 0.0)
        rhs.append(torch.as_tensor(f).cuda())
    insts = [Instance(h, w, kind, kind == "neumann") for h, w, kind in shapes]
    out = {}
    for mode in (1, 0):
        plan = PoissonPlan(insts, SolveParams(precision=precision, tolerance=1e-9,
                                              persistent_coarse=bool(mode), zero_start=True))
        plan.set_mask(2, torch.as_tensor(mask).cuda())
        plan.prepare()
        sols = []
        for _ in range(2):  # direct launches, then the solve graph
            x = [torch.empty_like(f) for f in rhs]
            res = plan.solve(rhs, x, scale=1.0)
            assert all(r.converged for r in res), res
            sols.append((x, [r.iterations for r in res]))
        plan.set_profiling(True)
        plan.solve(rhs, [torch.empty_like(f) for f in rhs], scale=1.0)
        kt = plan.kernel_times()
        assert (kt["coarse"]["launches"] > 0) == (mode == 1)
        assert (kt["bottom"]["launches"] > 0) == (mode == 0)
        plan.close()
        out[mode] = sols
    for (xa, ia), (xb, ib) in zip(out[0], out[1]):
        assert ia == ib
        for a, b in zip(xa, xb):
            assert torch.equal(a, b)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_dependent_launch_equals_serial_launch(precision):
    """Kernels launched as programmatic dependents (each waits for the one ahead
    before it touches the plan's mutable state) give bitwise the results of plain
    stream order, on an uneven batch of all boundary types, on direct launches,
    on the solve graph, with the persistent coarse launch and on the profiled path."""
    rng = np.random.default_rng(23)
    shapes = [(1030, 770, "neumann"), (513, 1201, "dirichlet"), (600, 640, "masked"),
              (257, 129, "neumann"), (40, 72, "dirichlet")]
    yy, xx = np.mgrid[0:600, 0:640]
    mask = ((yy - 300.0) ** 2 + (xx - 320.0) ** 2 < 250.0 ** 2).astype(np.uint8)
    rhs = []
    for h, w, kind in shapes:
        f = rng.standard_normal((h, w))
        if kind == "masked":
            f = np.where(mask, f, 0.0)
        rhs.append(torch.as_tensor(f).cuda())
    insts = [Instance(h, w, kind, kind == "neumann") for h, w, kind in shapes]
    out = {}
    for dep in (True, False):
        for persistent in (False, True):
            plan = PoissonPlan(insts, SolveParams(precision=precision, tolerance=1e-9,
                                                  dependent_launch=dep,
                                                  persistent_coarse=persistent,
                                                  zero_start=True))
            plan.set_mask(2, torch.as_tensor(mask).cuda())
            plan.prepare()
            sols = []
            for profiled in (False, False, False, True):  # direct, graph, graph, profiled
                plan.set_profiling(profiled)
                x = [torch.empty_like(f) for f in rhs]
                res = plan.solve(rhs, x, scale=1.0)
                assert all(r.converged for r in res), res
                sols.append((x, [r.iterations for r in res]))
            plan.close()
            out[(dep, persistent)] = sols
    ref = out[(False, False)]
    for key, sols in out.items():
        for (xa, ia), (xb, ib) in zip(ref, sols):
            assert ia == ib, key
            for a, b in zip(xa, xb):
                assert torch.equal(a, b), key


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_tile_shape_does_not_change_results(precision):
    """Level 1 of a 990 x 1000 instance (495 x 500 cells) has 128 large tiles: alone it
    runs on small tiles (fewer large tiles than SMs), in a batch of two on large
    tiles.  Every tile recomputes its halo exactly, so the solutions are bitwise the
    same either way, on direct launches and on the solve graph."""
    rng = np.random.default_rng(41)
    shapes = [(990, 1000, "neumann"), (1000, 980, "dirichlet")]
    rhs = [torch.as_tensor(rng.standard_normal(s[:2])).cuda() for s in shapes]
    params = SolveParams(precision=precision, tolerance=1e-9, zero_start=True)
    insts = [Instance(h, w, b, b == "neumann") for h, w, b in shapes]
    batch = PoissonPlan(insts, params)
    got = []
    for _ in range(2):
        xb = [torch.empty_like(r) for r in rhs]
        rb = batch.solve(rhs, xb, scale=1.0)
        got.append((xb, [r.iterations for r in rb]))
    batch.close()
    for k in range(len(shapes)):
        alone = PoissonPlan([insts[k]], params)
        for xb, its in got:
            xa = torch.empty_like(rhs[k])
            (ra,) = alone.solve([rhs[k]], [xa], scale=1.0)
            assert ra.converged and ra.iterations == its[k]
            assert torch.equal(xa, xb[k])
        alone.close()
