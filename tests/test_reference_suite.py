"""The reference's own test suite, run against the B200 drop-in.

Every case of gradient-domain/tests/test_solvers.py, test_operators.py and
test_applications.py (42 in all) is restated here with the reference's inputs
and bounds, calling ``gradient_domain_b200`` where the reference calls
``gradient_domain``.  The procedural images those tests draw from the
reference's synthetic.py (compositing, texture and radiance examples) come from
tests/golden/suite.npz, written by tests/golden/make_golden.py from the
reference itself; nothing here reads the reference checkout.

Where a case names a solver method, the drop-in runs that method on the GPU
(``direct`` is the FP64 B200 MGPCG to 1e-13, the others their device loops).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import gradient_domain_b200 as gd
from gradient_domain_b200.multigrid import _prolong, _restrict

pytestmark = pytest.mark.gpu

SUITE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "suite.npz")


@pytest.fixture(scope="module")
def suite():
    with np.load(SUITE) as data:
        return {k: data[k] for k in data.files}


# ---------------------------------------------------------------------------
# test_solvers.py


@pytest.mark.parametrize("method", ["direct", "cg", "multigrid", "mgcg"])
def test_every_solver_recovers_the_manufactured_solution(method):
    """test_solvers.py:24-31"""
    b, expected = gd.manufactured_problem((63, 63), seed=3)
    estimate, report = gd.solve_system(b, method=method, tolerance=1e-10)
    assert report.converged
    assert report.relative_residual < 1e-8
    assert np.abs(estimate - expected).max() < 1e-6


def test_solvers_agree_with_each_other():
    """test_solvers.py:34-39"""
    b, _ = gd.manufactured_problem((47, 61), seed=4)
    reference, _ = gd.solve_system(b, method="direct")
    for method in ("cg", "multigrid", "mgcg"):
        estimate, _ = gd.solve_system(b, method=method, tolerance=1e-11)
        assert np.abs(estimate - reference).max() < 1e-6


def test_unknown_method_is_rejected():
    """test_solvers.py:42-44"""
    with pytest.raises(KeyError):
        gd.solve_system(np.zeros((8, 8)), method="jacobi")


def test_zero_right_hand_side_gives_zero():
    """test_solvers.py:47-50"""
    estimate, report = gd.solve_system(np.zeros((16, 16)), method="mgcg")
    assert np.allclose(estimate, 0.0)
    assert report.relative_residual == 0.0


@pytest.mark.parametrize("size", [31, 63, 127, 255])
def test_multigrid_convergence_does_not_depend_on_the_grid(size):
    """test_solvers.py:53-59"""
    b, _ = gd.manufactured_problem((size, size), seed=5)
    _, report = gd.solve(b, options=gd.MultigridOptions(tolerance=1e-10))
    assert report.converged
    assert report.cycles <= 10
    assert report.convergence_factor < 0.1


def test_restriction_is_the_scaled_adjoint_of_prolongation():
    """test_solvers.py:63-73"""
    rng = np.random.default_rng(6)
    fine_shape = (31, 25)
    coarse_shape = ((fine_shape[0] - 1) // 2, (fine_shape[1] - 1) // 2)
    fine = rng.standard_normal(fine_shape)
    coarse = rng.standard_normal(coarse_shape)
    left = float(np.sum(_restrict(fine) * coarse))
    right = 0.25 * float(np.sum(fine * _prolong(coarse, fine_shape)))
    assert left == pytest.approx(right, rel=1e-12)


def test_prolongation_reproduces_a_constant_in_the_interior():
    """test_solvers.py:76-81: zeros outside the coarse grid, so only the interior
    (complete stencils) reaches the constant."""
    fine = _prolong(np.ones((7, 7)), (15, 15))
    assert np.allclose(fine[1:-1, 1:-1], 1.0)


def test_one_cycle_reduces_the_residual_by_an_order_of_magnitude():
    """test_solvers.py:84-87"""
    b, _ = gd.manufactured_problem((127, 127), seed=7)
    _, report = gd.solve(b, options=gd.MultigridOptions(max_cycles=1, tolerance=0.0))
    assert report.residuals[1] < 0.1 * report.residuals[0]


def test_neumann_solver_is_exact():
    """test_solvers.py:90-101"""
    rng = np.random.default_rng(8)
    for shape in ((64, 64), (97, 131)):
        expected = rng.standard_normal(shape)
        expected -= expected.mean()
        padded = np.pad(expected, 1, mode="edge")
        b = (padded[:-2, 1:-1] + padded[2:, 1:-1] + padded[1:-1, :-2] + padded[1:-1, 2:]
             - 4.0 * expected)
        assert np.abs(gd.solve_neumann(b) - expected).max() < 1e-10


def test_neumann_solution_has_zero_mean():
    """test_solvers.py:104-107"""
    rng = np.random.default_rng(9)
    b = rng.standard_normal((32, 40))
    b -= b.mean()
    assert abs(float(gd.solve_neumann(b).mean())) < 1e-12


def test_residual_matches_the_operator():
    """test_solvers.py:111-114"""
    b, _ = gd.manufactured_problem((33, 33), seed=10)
    estimate, report = gd.solve_system(b, method="mgcg", tolerance=1e-9)
    residual = float(np.linalg.norm(b - gd.laplacian(estimate))) / float(np.linalg.norm(b))
    assert residual == pytest.approx(report.relative_residual, rel=1e-9)


# ---------------------------------------------------------------------------
# test_operators.py


@pytest.fixture
def rng():
    return np.random.default_rng(11)


def test_divergence_is_the_negative_adjoint_of_the_gradient(rng):
    """test_operators.py:28-36"""
    u = rng.standard_normal((23, 31))
    vx, vy = rng.standard_normal((23, 31)), rng.standard_normal((23, 31))
    gx, gy = gd.gradient(u)
    left = float(np.sum(gx * vx) + np.sum(gy * vy))
    right = -float(np.sum(u * gd.divergence(vx, vy)))
    assert left == pytest.approx(right, rel=1e-12)


def test_gradient_of_a_constant_vanishes():
    """test_operators.py:39-42"""
    gx, gy = gd.gradient(np.full((9, 12), 3.5))
    assert np.allclose(gx, 0.0) and np.allclose(gy, 0.0)


def test_gradient_reproduces_a_linear_ramp():
    """test_operators.py:45-49"""
    rows, columns = np.mgrid[0:8, 0:10]
    gx, gy = gd.gradient(2.0 * columns + 3.0 * rows)
    assert np.allclose(gx[:, :-1], 2.0)
    assert np.allclose(gy[:-1, :], 3.0)


def test_composition_is_the_neumann_laplacian(rng):
    """test_operators.py:52-58"""
    u = rng.standard_normal((17, 21))
    padded = np.pad(u, 1, mode="edge")
    expected = (padded[:-2, 1:-1] + padded[2:, 1:-1] + padded[1:-1, :-2] + padded[1:-1, 2:]
                - 4.0 * u)
    assert np.allclose(gd.divergence(*gd.gradient(u)), expected)


def test_dense_and_sparse_laplacians_agree(rng):
    """test_operators.py:61-66"""
    u = rng.standard_normal((13, 19))
    for spacing in (1.0, 0.5, 2.0):
        expected = gd.laplacian(u, spacing)
        actual = (gd.sparse_laplacian(u.shape, spacing) @ u.reshape(-1)).reshape(u.shape)
        assert np.allclose(actual, expected)


def test_laplacian_is_symmetric_negative_definite():
    """test_operators.py:69-72"""
    operator = gd.sparse_laplacian((7, 9)).toarray()
    assert np.allclose(operator, operator.T)
    assert np.linalg.eigvalsh(operator).max() < 0.0


def test_folding_the_boundary_reproduces_the_full_stencil(rng):
    """test_operators.py:75-81"""
    full = rng.standard_normal((14, 18))
    interior = full[1:-1, 1:-1]
    padded_result = gd.laplacian(full)[1:-1, 1:-1]
    folded = gd.laplacian(interior) - gd.fold_boundary(np.zeros_like(interior), full)
    assert np.allclose(folded, padded_result)


def test_folding_scales_with_the_grid_spacing():
    """test_operators.py:84-90: corners lose two neighbours, edges one, the centre none."""
    folded = gd.fold_boundary(np.zeros((3, 3)), np.ones((5, 5)), spacing=0.5)
    assert folded[0, 0] == pytest.approx(-8.0)
    assert folded[0, 1] == pytest.approx(-4.0)
    assert folded[1, 1] == pytest.approx(0.0)


# ---------------------------------------------------------------------------
# test_applications.py


class Example:
    """The compositing example of test_applications.py:32-34 (synthetic.py's
    make_compositing_example(shape=(160, 240), seed=0))."""

    def __init__(self, s):
        self.target, self.source, self.mask = s["ex_target"], s["ex_source"], s["ex_mask"]
        self.offset = tuple(int(v) for v in s["ex_offset"])
        self._naive = s["ex_naive"]

    def naive_composite(self):
        return self._naive.copy()

    def placed(self):
        placed = np.zeros(self.target.shape[:2], dtype=bool)
        row, column = self.offset
        height, width = self.source.shape[:2]
        placed[row:row + height, column:column + width] = self.mask
        return placed


@pytest.fixture(scope="module")
def example(suite):
    return Example(suite)


def _decades(image):
    """Log ratio of the 99th to the 1st luminance percentile (test_applications.py:37-41)."""
    luminance = np.maximum(image @ np.array([0.2126, 0.7152, 0.0722]), 1e-8)
    low, high = np.percentile(luminance, [1, 99])
    return float(np.log10(max(high, 1e-8) / max(low, 1e-8)))


def _disc(shape, radius):
    rows, columns = np.mgrid[0:shape[0], 0:shape[1]]
    centre = (shape[0] / 2, shape[1] / 2)
    return (rows - centre[0]) ** 2 + (columns - centre[1]) ** 2 < radius ** 2


def test_integrating_an_image_reproduces_it():
    """test_applications.py:49-55"""
    image = np.random.default_rng(0).random((40, 52, 3))
    result, reports = gd.solve_dirichlet(gd.GuidanceField.of(image), image, method="direct")
    assert np.abs(result - image).max() < 1e-9
    assert len(reports) == 3


def test_cloning_an_image_into_itself_changes_nothing(example):
    """test_applications.py:58-62"""
    mask = _disc(example.target.shape[:2], 30.0)
    result, _ = gd.solve_masked(gd.GuidanceField.of(example.target), example.target, mask)
    assert np.abs(result - example.target).max() < 1e-9


def test_masked_domain_leaves_the_destination_untouched(example):
    """test_applications.py:65-74"""
    result, _ = gd.seamless_clone(example.source, example.target, example.mask, example.offset,
                                  domain="mask")
    placed = example.placed()
    assert np.array_equal(result[~placed], example.target[~placed])


def test_the_two_formulations_agree_up_to_a_harmonic_correction(example):
    """test_applications.py:77-87"""
    masked, _ = gd.seamless_clone(example.source, example.target, example.mask, example.offset,
                                  domain="mask")
    rectangle, _ = gd.seamless_clone(example.source, example.target, example.mask,
                                     example.offset, domain="rectangle", method="direct")
    difference = np.abs(masked - rectangle)
    assert difference.mean() < 5e-3
    assert difference.max() < 0.2


def _boundary_ring(mask):
    """Pixels where the mask changes value (test_applications.py:90-102)."""
    height, width = mask.shape
    padded = np.pad(mask, 1)
    dilated = np.zeros_like(mask)
    eroded = np.ones_like(mask)
    for dr, dc in ((0, 1), (0, -1), (1, 0), (-1, 0), (0, 0)):
        shifted = padded[1 + dr:1 + dr + height, 1 + dc:1 + dc + width]
        dilated |= shifted
        eroded &= shifted
    return dilated & ~eroded


def test_cloning_removes_the_seam_that_copying_leaves(example):
    """test_applications.py:105-121: seam energy drops more than four times."""
    naive = example.naive_composite()
    blended, _ = gd.seamless_clone(example.source, example.target, example.mask, example.offset,
                                   domain="mask")
    ring = _boundary_ring(example.placed())

    def seam_energy(image):
        gradient_magnitude = np.abs(np.diff(image, axis=0)).mean(axis=2)
        return float(gradient_magnitude[ring[:-1]].mean())

    assert seam_energy(blended) < 0.25 * seam_energy(naive)


@pytest.mark.parametrize("mode", ["import", "mixed", "average"])
def test_every_blend_mode_runs(example, mode):
    """test_applications.py:124-130"""
    result, _ = gd.seamless_clone(example.source, example.target, example.mask, example.offset,
                                  mode=mode, domain="mask")
    assert result.shape == example.target.shape
    assert np.isfinite(result).all()


def test_unknown_mode_and_domain_are_rejected(example):
    """test_applications.py:133-139"""
    with pytest.raises(ValueError):
        gd.seamless_clone(example.source, example.target, example.mask, example.offset,
                          mode="blend")
    with pytest.raises(ValueError):
        gd.seamless_clone(example.source, example.target, example.mask, example.offset,
                          domain="triangle")


def test_patch_outside_the_target_is_rejected(example):
    """test_applications.py:142-146"""
    with pytest.raises(ValueError):
        gd.seamless_clone(example.source, example.target, example.mask, offset=(10_000, 0),
                          domain="mask")


def test_flattening_with_every_edge_retained_is_the_identity(suite):
    """test_applications.py:149-152"""
    image = suite["tex96_image"]
    result, _ = gd.texture_flatten(image, np.ones(image.shape[:2]), method="direct")
    assert np.abs(result - image).max() < 1e-9


def test_flattening_reduces_texture_energy(suite):
    """test_applications.py:155-164"""
    image, edges = suite["tex128_image"], suite["tex128_edges"]
    flattened, _ = gd.texture_flatten(image, edges, method="mgcg")

    def texture_energy(candidate):
        interior = ~edges.astype(bool)
        variation = np.abs(np.diff(candidate, axis=1)).mean(axis=2)
        return float(variation[interior[:, :-1]].mean())

    assert texture_energy(flattened) < 0.2 * texture_energy(image)


def test_illumination_change_lifts_a_dark_selection():
    """test_applications.py:167-175"""
    _, columns = np.mgrid[0:96, 0:96]
    image = np.repeat((0.05 + 0.02 * np.sin(columns * 0.4))[..., None], 3, axis=2)
    mask = _disc((96, 96), 30.0)
    result, _ = gd.illumination_change(image, mask, alpha=0.4, beta=0.6)
    interior = mask & ~_disc((96, 96), 24.0)
    assert result[interior].std() > image[interior].std()
    assert np.array_equal(result[~mask], image[~mask])


def test_tone_mapping_compresses_the_dynamic_range(suite):
    """test_applications.py:178-188"""
    radiance = suite["rad128x176"]
    mapped, factor = gd.tone_map(radiance)
    assert mapped.shape == radiance.shape
    assert mapped.min() >= 0.0 and mapped.max() <= 1.0
    assert factor.shape == radiance.shape[:2]
    assert _decades(mapped) < 0.4 * _decades(radiance)


def test_smaller_beta_compresses_more(suite):
    """test_applications.py:191-198"""
    radiance = suite["rad96x128"]
    gentle, _ = gd.tone_map(radiance, gd.ToneMapConfig(beta=0.95))
    strong, _ = gd.tone_map(radiance, gd.ToneMapConfig(beta=0.4))
    assert _decades(strong) < _decades(gentle)


def test_attenuation_leaves_a_flat_image_alone():
    """test_applications.py:201-204"""
    factor = gd.attenuation_field(np.zeros((64, 64)), gd.ToneMapConfig())
    assert np.isfinite(factor).all()
    assert factor.min() > 0.0


def test_tone_mapping_rejects_a_grayscale_input():
    """test_applications.py:207-209"""
    with pytest.raises(ValueError):
        gd.tone_map(np.ones((16, 16)))
