"""Pin the CPU oracle to the reference: golden vectors and the reference's own tests.

The oracle is the checker for every GPU parity test, so it is itself checked
here against outputs of the reference package (tests/golden/golden.npz) and
against the known answers asserted by gradient-domain/tests/*.py.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import hdr, multigrid, operators, poisson, solvers


def _manufactured(shape, seed):
    """Manufactured problem of gradient-domain/src/gradient_domain/benchmark.py:65-95."""
    rng = np.random.default_rng(seed)
    rows, cols = np.mgrid[0:shape[0], 0:shape[1]] / max(shape)
    sol = (np.sin(3.0 * np.pi * cols) * np.sin(2.0 * np.pi * rows)
           + 0.4 * np.cos(11.0 * np.pi * cols) * np.sin(7.0 * np.pi * rows)
           + 0.25 * rng.standard_normal(shape))
    sol[0] = sol[-1] = 0.0
    sol[:, 0] = sol[:, -1] = 0.0
    return operators.laplacian(sol), sol


def test_manufactured_matches_golden(golden):
    b, exact = _manufactured((47, 61), 4)
    np.testing.assert_array_equal(b, golden["sys_b"])
    np.testing.assert_array_equal(exact, golden["sys_exact"])


def test_operators_match_golden(golden):
    gx, gy = operators.gradient(golden["op_u"])
    np.testing.assert_array_equal(gx, golden["op_gx"])
    np.testing.assert_array_equal(gy, golden["op_gy"])
    np.testing.assert_array_equal(operators.divergence(golden["op_vx"], golden["op_vy"]),
                                  golden["op_div"])
    np.testing.assert_array_equal(operators.laplacian(golden["op_u"], 0.5), golden["op_lap_h05"])
    np.testing.assert_array_equal(
        operators.fold_boundary(np.zeros((12, 16)), golden["op_ring"], 0.5), golden["op_fold"])


@pytest.mark.parametrize("name", ["vc63", "vc47x61", "vc30x22", "vc8"])
def test_v_cycle_matches_golden(golden, name):
    pre, post, cs, sweeps, h = golden[f"{name}_opts"]
    opts = multigrid.MultigridOptions(int(pre), int(post), int(cs), int(sweeps))
    b = golden[f"{name}_b"]
    for start, key in ((np.zeros_like(b), "zero"), (golden[f"{name}_u0"], "warm")):
        got = multigrid.v_cycle(start, b, float(h), opts)
        ref = golden[f"{name}_{key}"]
        assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


SMOOTH_CASES = ["sm37x53", "sm37x53s3", "sm5x131", "sm70x260s6"]


@pytest.mark.parametrize("name", SMOOTH_CASES)
def test_smooth_matches_golden_bitwise(golden, name):
    sweeps, h = golden[f"{name}_opts"]
    u0, b = golden[f"{name}_u0"], golden[f"{name}_b"]
    got64 = multigrid.smooth(u0, b, float(h), int(sweeps))
    got32 = multigrid.smooth(u0.astype(np.float32), b.astype(np.float32), float(h), int(sweeps))
    assert got32.dtype == np.float32
    np.testing.assert_array_equal(got64, golden[f"{name}_f64"])
    np.testing.assert_array_equal(got32, golden[f"{name}_f32"])


def test_transfers_match_golden(golden):
    np.testing.assert_allclose(multigrid.restrict(golden["tr_fine"]), golden["tr_restrict"],
                               rtol=0, atol=1e-14)
    np.testing.assert_allclose(multigrid.prolong(golden["tr_coarse"], (31, 25)),
                               golden["tr_prolong"], rtol=0, atol=1e-14)


def test_multigrid_solve_history_matches_golden(golden):
    u, rep = multigrid.solve(golden["mgsolve_b"],
                             options=multigrid.MultigridOptions(tolerance=1e-10))
    np.testing.assert_allclose(rep.residuals, golden["mgsolve_hist"], rtol=1e-9)
    assert np.abs(u - golden["mgsolve_u"]).max() < 1e-12


@pytest.mark.parametrize("method", ["direct", "cg", "multigrid", "mgcg"])
def test_solve_system_matches_golden(golden, method):
    u, rep = solvers.solve_system(golden["sys_b"], method=method, tolerance=1e-10)
    its, res, conv = golden[f"sys_{method}_info"]
    assert rep.iterations == int(its)
    assert bool(conv) == rep.converged
    assert np.abs(u - golden[f"sys_{method}_u"]).max() < 1e-10


@pytest.mark.parametrize("key", ["neu32x40", "neu97x131", "neu64x64"])
def test_solve_neumann_matches_golden(golden, key):
    np.testing.assert_allclose(solvers.solve_neumann(golden[f"{key}_b"]), golden[f"{key}_u"],
                               rtol=0, atol=1e-12)


def test_applications_match_golden(golden):
    field = poisson.GuidanceField.of(golden["app_src"])
    got, reps = poisson.solve_masked(field, golden["app_img"], golden["app_disc"])
    assert np.abs(got - golden["app_masked"]).max() < 1e-12 and len(reps) == 3
    got, _ = poisson.solve_dirichlet(field, golden["app_img"], method="direct")
    assert np.abs(got - golden["app_dirichlet"]).max() < 1e-12
    off = tuple(int(v) for v in golden["clone_offset"])
    for mode in ("import", "mixed", "average"):
        got, _ = poisson.seamless_clone(golden["clone_source"], golden["clone_target"],
                                        golden["clone_mask"], off, mode=mode, domain="mask")
        assert np.abs(got - golden[f"clone_{mode}_mask"]).max() < 1e-12
    got, _ = poisson.seamless_clone(golden["clone_source"], golden["clone_target"],
                                    golden["clone_mask"], off, domain="rectangle",
                                    method="direct")
    assert np.abs(got - golden["clone_import_rect"]).max() < 1e-12
    got, _ = poisson.texture_flatten(golden["tex_image"], golden["tex_edges"], method="direct")
    assert np.abs(got - golden["tex_flat"]).max() < 1e-12
    got, _ = poisson.illumination_change(golden["tex_image"], golden["illum_mask"],
                                         alpha=0.4, beta=0.6)
    assert np.abs(got - golden["illum"]).max() < 1e-12


def test_tone_map_matches_golden(golden):
    mapped, factor = hdr.tone_map(golden["tm_radiance"])
    np.testing.assert_allclose(factor, golden["tm_factor"], rtol=1e-12)
    np.testing.assert_allclose(mapped, golden["tm_mapped"], rtol=0, atol=1e-12)
    lum = np.log(np.maximum(golden["tm_radiance"] @ hdr.LUMA, np.finfo(float).tiny))
    np.testing.assert_allclose(
        hdr.attenuation_field(lum, hdr.ToneMapConfig(alpha=0.1, beta=0.85, levels=1)),
        golden["att_levels1"], rtol=1e-12)


# Known answers asserted by the reference's own suite, restated on the oracle.

@pytest.mark.parametrize("method", ["direct", "cg", "multigrid", "mgcg"])
def test_every_solver_recovers_manufactured_solution(method):
    # gradient-domain/tests/test_solvers.py:24-31
    b, exact = _manufactured((63, 63), 3)
    u, rep = solvers.solve_system(b, method=method, tolerance=1e-10)
    assert rep.converged and rep.relative_residual < 1e-8
    assert np.abs(u - exact).max() < 1e-6


def test_unknown_method_and_zero_rhs():
    # gradient-domain/tests/test_solvers.py:42-50
    with pytest.raises(KeyError):
        solvers.solve_system(np.zeros((8, 8)), method="jacobi")
    u, rep = solvers.solve_system(np.zeros((16, 16)))
    assert np.allclose(u, 0.0) and rep.relative_residual == 0.0


@pytest.mark.parametrize("size", [31, 63, 127])
def test_multigrid_grid_independent(size):
    # gradient-domain/tests/test_solvers.py:53-59
    b, _ = _manufactured((size, size), 5)
    _, rep = multigrid.solve(b, options=multigrid.MultigridOptions(tolerance=1e-10))
    assert rep.converged and rep.cycles <= 10 and rep.convergence_factor < 0.1


def test_restriction_is_scaled_adjoint():
    # gradient-domain/tests/test_solvers.py:63-73
    rng = np.random.default_rng(6)
    f, c = rng.standard_normal((31, 25)), rng.standard_normal((15, 12))
    assert float(np.sum(multigrid.restrict(f) * c)) == pytest.approx(
        0.25 * float(np.sum(f * multigrid.prolong(c, (31, 25)))), rel=1e-12)


def test_neumann_exact_and_zero_mean():
    # gradient-domain/tests/test_solvers.py:90-107
    rng = np.random.default_rng(8)
    for shape in ((64, 64), (97, 131)):
        x = rng.standard_normal(shape)
        x -= x.mean()
        assert np.abs(solvers.solve_neumann(operators.neumann_laplacian(x)) - x).max() < 1e-10
    b = np.random.default_rng(9).standard_normal((32, 40))
    b -= b.mean()
    assert abs(float(solvers.solve_neumann(b).mean())) < 1e-12


def test_operator_adjointness_and_folding():
    # gradient-domain/tests/test_operators.py:28-90
    rng = np.random.default_rng(11)
    u = rng.standard_normal((23, 31))
    vx, vy = rng.standard_normal((23, 31)), rng.standard_normal((23, 31))
    gx, gy = operators.gradient(u)
    assert float(np.sum(gx * vx) + np.sum(gy * vy)) == pytest.approx(
        -float(np.sum(u * operators.divergence(vx, vy))), rel=1e-12)
    w = rng.standard_normal((17, 21))
    assert np.allclose(operators.divergence(*operators.gradient(w)),
                       operators.neumann_laplacian(w))
    full = rng.standard_normal((14, 18))
    inner = full[1:-1, 1:-1]
    assert np.allclose(operators.laplacian(inner) - operators.fold_boundary(np.zeros_like(inner),
                                                                           full),
                       operators.laplacian(full)[1:-1, 1:-1])


@pytest.mark.parametrize("key", ["mp63x63s3", "mp47x61s4", "mp127x127s7", "mp33x33s10",
                                 "mp31x31s5"])
def test_package_manufactured_problem_matches_reference(key):
    """The package's benchmark.manufactured_problem (the known-answer generator the
    reference's solver tests use) against the reference's own output."""
    import os

    from gradient_domain_b200.benchmark import manufactured_problem
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "suite.npz")
    shape_s, seed = key[2:].split("s")
    shape = tuple(int(v) for v in shape_s.split("x"))
    with np.load(path) as data:
        np.testing.assert_array_equal(manufactured_problem(shape, seed=int(seed))[0], data[key])
