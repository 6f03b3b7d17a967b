"""CPU checks of the cell-centred multigrid design (through the NumPy model).

The GPU kernels are compared with this model in the gpu-marked tests; here the
model itself is checked: it solves each boundary type to the reference's
answer, its V-cycle is symmetric (so plain PCG is valid), and its iteration
count does not grow with the grid.
"""

from __future__ import annotations

import numpy as np
import pytest

import mg_model as M
from oracle import operators, poisson, solvers


@pytest.mark.parametrize("boundary", ["neumann", "dirichlet"])
def test_vcycle_is_symmetric(boundary):
    rng = np.random.default_rng(1)
    levels = M.build_levels((70, 90), boundary)
    a, b = rng.standard_normal((70, 90)), rng.standard_normal((70, 90))
    if boundary == "neumann":
        a -= a.mean()
        b -= b.mean()
    left = np.sum(a * M.vcycle(levels, b))
    right = np.sum(b * M.vcycle(levels, a))
    assert left == pytest.approx(right, rel=1e-12)


def test_neumann_model_matches_dct_oracle():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((97, 131))
    x -= x.mean()
    b = operators.neumann_laplacian(x)
    u, _ = M.mgpcg(-b, "neumann", tol=1e-13)
    u -= u.mean()
    assert np.abs(u - solvers.solve_neumann(b)).max() < 1e-9


def test_dirichlet_model_matches_direct_oracle():
    rng = np.random.default_rng(3)
    b = rng.standard_normal((47, 61))
    u, _ = M.mgpcg(-b, "dirichlet", tol=1e-13)
    ref, _, _ = solvers.solve_direct(b, 1.0, 0.0, 0)
    assert np.abs(u - ref).max() < 1e-9


def test_masked_model_matches_splu_oracle():
    rng = np.random.default_rng(4)
    yy, xx = np.mgrid[0:60, 0:70]
    mask = (yy - 30.0) ** 2 + (xx - 33.0) ** 2 < 24.0 ** 2
    img = rng.random((60, 70))
    field = poisson.GuidanceField.of(rng.random((60, 70)))
    ref, _ = poisson.solve_masked(field, img, mask)
    interior, index, _ = poisson.masked_system(mask)
    rhs = poisson.masked_rhs(operators.divergence(field.gx, field.gy), img, interior, index)
    f = np.zeros(mask.shape)
    f[interior] = -rhs
    u, _ = M.mgpcg(f, "masked", interior, tol=1e-13)
    got = img.copy()
    got[interior] = u[interior]
    assert np.abs(got - ref).max() < 1e-9


def test_iterations_do_not_grow_with_the_grid():
    rng = np.random.default_rng(5)
    counts = [M.mgpcg(rng.standard_normal((n, n)), "neumann")[1] for n in (64, 128, 256, 512)]
    assert max(counts) <= 9
