"""The reference's Dirichlet solvers and DCT Neumann solver, restated (oracle).

Follows ``gradient-domain/src/gradient_domain/solvers.py``.  Every iterative
method works on the SPD system -L u = -b (lines 29-31).
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import scipy.sparse.linalg as spla
from scipy.fft import dctn, idctn

from .multigrid import MultigridOptions, v_cycle
from .operators import laplacian, sparse_laplacian


@dataclass
class SolverReport:
    """gradient-domain/src/gradient_domain/solvers.py:50-75."""

    method: str
    iterations: int
    relative_residual: float
    seconds: float
    converged: bool


def relative_residual(u, b, spacing):
    """gradient-domain/src/gradient_domain/solvers.py:78-82."""
    scale = float(np.linalg.norm(b))
    return 0.0 if scale == 0.0 else float(np.linalg.norm(b - laplacian(u, spacing))) / scale


def solve_direct(b, spacing, tolerance, max_iterations):
    """SuperLU on the assembled operator, gradient-domain/src/gradient_domain/solvers.py:85-90."""
    lu = spla.splu(sparse_laplacian(b.shape, spacing).tocsc())
    return lu.solve(b.ravel()).reshape(b.shape), 0, True


def _pcg(b, spacing, tolerance, max_iterations, precondition):
    """Shared PCG loop of gradient-domain/src/gradient_domain/solvers.py:99-118 and :142-160."""
    rhs = -b
    u = np.zeros_like(b)
    r = rhs.copy()
    p = precondition(r)
    rz = float(np.sum(r * p))
    target = tolerance * float(np.linalg.norm(rhs))
    for it in range(1, max_iterations + 1):
        q = -laplacian(p, spacing)
        alpha = rz / float(np.sum(p * q))
        u += alpha * p
        r -= alpha * q
        if float(np.linalg.norm(r)) <= target:
            return u, it, True
        z = precondition(r)
        rz_new = float(np.sum(r * z))
        p = z + (rz_new / rz) * p
        rz = rz_new
    return u, max_iterations, False


def solve_cg(b, spacing, tolerance, max_iterations):
    """Jacobi-PCG, gradient-domain/src/gradient_domain/solvers.py:93-118."""
    diag = 4.0 / (spacing * spacing)
    return _pcg(b, spacing, tolerance, max_iterations, lambda r: r / diag)


def solve_multigrid(b, spacing, tolerance, max_iterations):
    """Stand-alone V-cycles, gradient-domain/src/gradient_domain/solvers.py:121-131."""
    options = MultigridOptions(max_cycles=max_iterations, tolerance=tolerance)
    u = np.zeros_like(b)
    scale = float(np.linalg.norm(b)) or 1.0
    for cycle in range(1, max_iterations + 1):
        u = v_cycle(u, b, spacing, options)
        if float(np.linalg.norm(b - laplacian(u, spacing))) / scale < tolerance:
            return u, cycle, True
    return u, max_iterations, False


def solve_mgcg(b, spacing, tolerance, max_iterations):
    """PCG with one V-cycle (pre = post = 1) as preconditioner,
    gradient-domain/src/gradient_domain/solvers.py:134-160."""
    options = MultigridOptions(pre_smoothing=1, post_smoothing=1)
    return _pcg(b, spacing, tolerance, max_iterations,
                lambda r: v_cycle(np.zeros_like(r), -r, spacing, options))


SOLVERS = {"direct": solve_direct, "cg": solve_cg, "multigrid": solve_multigrid,
           "mgcg": solve_mgcg}


def solve_system(b, method="mgcg", spacing=1.0, tolerance=1e-8, max_iterations=2000):
    """Front door, gradient-domain/src/gradient_domain/solvers.py:171-221."""
    if method not in SOLVERS:
        raise KeyError(method)
    b = np.asarray(b, dtype=float)
    if not np.any(b):
        return np.zeros_like(b), SolverReport(method, 0, 0.0, 0.0, True)
    t0 = time.perf_counter()
    u, its, ok = SOLVERS[method](b, spacing, tolerance, max_iterations)
    return u, SolverReport(method, its, relative_residual(u, b, spacing),
                           time.perf_counter() - t0, ok)


def neumann_eigenvalues(rows, cols):
    """Eigenvalues of the edge-replicated Laplacian under DCT-II,
    gradient-domain/src/gradient_domain/solvers.py:253-258."""
    return (2.0 * np.cos(np.pi * np.arange(rows) / rows)[:, None]
            + 2.0 * np.cos(np.pi * np.arange(cols) / cols)[None, :] - 4.0)


def solve_neumann(b, workers=None):
    """Zero-mean DCT solve, gradient-domain/src/gradient_domain/solvers.py:224-262."""
    b = np.asarray(b, dtype=float)
    lam = neumann_eigenvalues(*b.shape)
    lam[0, 0] = 1.0
    coeffs = dctn(b, type=2, norm="ortho", workers=workers) / lam
    coeffs[0, 0] = 0.0
    return idctn(coeffs, type=2, norm="ortho", workers=workers)
