"""Vertex-centred geometric multigrid of the reference, restated (oracle).

Follows ``gradient-domain/src/gradient_domain/multigrid.py``: interior grid
(m, n) with zero Dirichlet values outside, coarsening m -> (m - 1) // 2 with
coarse point I on fine point 2I + 1, red-black Gauss-Seidel with colour
(i + j) % 2 == 0 first in every sweep, full-weighting restriction P^T / 4 and
bilinear prolongation P, 60 sweeps on the coarsest grid.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .operators import laplacian, neighbour_sum


@dataclass
class MultigridOptions:
    """Defaults of gradient-domain/src/gradient_domain/multigrid.py:47-71."""

    pre_smoothing: int = 2
    post_smoothing: int = 2
    coarsest_size: int = 8
    coarsest_sweeps: int = 60
    max_cycles: int = 60
    tolerance: float = 1e-8


@dataclass
class MultigridReport:
    """gradient-domain/src/gradient_domain/multigrid.py:75-108."""

    residuals: list = field(default_factory=list)
    cycles: int = 0
    converged: bool = False

    @property
    def convergence_factor(self):
        if len(self.residuals) < 2 or self.residuals[0] <= 0:
            return float("nan")
        return float((self.residuals[-1] / self.residuals[0]) ** (1.0 / (len(self.residuals) - 1)))


def coarse_shape(shape):
    """gradient-domain/src/gradient_domain/multigrid.py:143-144."""
    return ((shape[0] - 1) // 2, (shape[1] - 1) // 2)


def prolong_1d_weights(fine, coarse):
    """Dense 1-D interpolation matrix, gradient-domain/src/gradient_domain/multigrid.py:111-133.

    Odd fine index i takes coarse (i-1)/2 with weight 1; even fine index takes
    coarse i/2 - 1 and i/2 with weight 1/2 each; out-of-range coarse indices are
    the homogeneous Dirichlet value and contribute nothing.
    """
    p = np.zeros((fine, coarse))
    for i in range(fine):
        if i % 2:
            src = (i - 1) // 2
            if 0 <= src < coarse:
                p[i, src] = 1.0
        else:
            for src in (i // 2 - 1, i // 2):
                if 0 <= src < coarse:
                    p[i, src] = 0.5
    return p


def smooth(u, b, spacing, sweeps):
    """Red-black Gauss-Seidel, gradient-domain/src/gradient_domain/multigrid.py:147-165."""
    h2 = spacing * spacing
    rows = np.arange(u.shape[0])[:, None]
    cols = np.arange(u.shape[1])[None, :]
    colour = (rows + cols) % 2
    for _ in range(sweeps):
        for parity in (0, 1):
            candidate = 0.25 * (neighbour_sum(u) - h2 * b)
            u = np.where(colour == parity, candidate, u)
    return u


def restrict(residual):
    """Full weighting (1/4) Rows^T r Cols, gradient-domain/src/gradient_domain/multigrid.py:169-174."""
    m, n = residual.shape
    mc, nc = coarse_shape((m, n))
    return (prolong_1d_weights(m, mc).T @ residual @ prolong_1d_weights(n, nc)) * 0.25


def prolong(correction, shape):
    """Bilinear Rows e Cols^T, gradient-domain/src/gradient_domain/multigrid.py:177-181."""
    rows = prolong_1d_weights(shape[0], correction.shape[0])
    cols = prolong_1d_weights(shape[1], correction.shape[1])
    return rows @ correction @ cols.T


def v_cycle(u, b, spacing, options):
    """gradient-domain/src/gradient_domain/multigrid.py:184-215."""
    cs = coarse_shape(u.shape)
    if min(u.shape) <= options.coarsest_size or min(cs) < 2:
        return smooth(u, b, spacing, options.coarsest_sweeps)
    u = smooth(u, b, spacing, options.pre_smoothing)
    r = b - laplacian(u, spacing)
    e = v_cycle(np.zeros(cs), restrict(r), 2.0 * spacing, options)
    u = u + prolong(e, u.shape)
    return smooth(u, b, spacing, options.post_smoothing)


def solve(b, spacing=1.0, options=None, initial=None):
    """Repeated V-cycles, gradient-domain/src/gradient_domain/multigrid.py:218-255."""
    options = options or MultigridOptions()
    b = np.asarray(b, dtype=float)
    u = np.zeros_like(b) if initial is None else np.array(initial, dtype=float)
    scale = float(np.linalg.norm(b))
    if scale == 0.0:
        return u, MultigridReport([0.0], 0, True)
    history = [float(np.linalg.norm(b - laplacian(u, spacing))) / scale]
    for cycle in range(1, options.max_cycles + 1):
        u = v_cycle(u, b, spacing, options)
        history.append(float(np.linalg.norm(b - laplacian(u, spacing))) / scale)
        if history[-1] < options.tolerance:
            return u, MultigridReport(history, cycle, True)
    return u, MultigridReport(history, options.max_cycles, False)
