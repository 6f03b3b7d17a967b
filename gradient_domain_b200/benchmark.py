"""Solver scaling study on the GPU solvers.

Same interface as gradient-domain/src/gradient_domain/benchmark.py:
``manufactured_problem`` (:65-95) builds a right-hand side with a known
solution (smooth modes plus white noise, zero Dirichlet ring), and
``solver_scaling`` (:98-149) times every method of ``SOLVERS`` on it.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .solvers import solve_system

__all__ = ["BenchmarkRecord", "BenchmarkTable", "manufactured_problem", "solver_scaling"]


@dataclass
class BenchmarkRecord:
    method: str
    shape: tuple
    unknowns: int
    seconds: float
    iterations: int
    relative_residual: float
    max_error: float

    def as_dict(self) -> dict:
        return {"method": self.method, "shape": list(self.shape), "unknowns": self.unknowns,
                "seconds": self.seconds, "iterations": self.iterations,
                "relative_residual": self.relative_residual, "max_error": self.max_error}


def _five_point(u: np.ndarray) -> np.ndarray:
    p = np.pad(u, 1)
    return p[:-2, 1:-1] + p[2:, 1:-1] + p[1:-1, :-2] + p[1:-1, 2:] - 4.0 * u


def manufactured_problem(shape, seed: int = 0):
    """Right-hand side ``b`` and exact solution of ``laplacian(u) = b``."""
    rng = np.random.default_rng(seed)
    rows, cols = np.mgrid[0:shape[0], 0:shape[1]] / max(shape)
    solution = (np.sin(3.0 * np.pi * cols) * np.sin(2.0 * np.pi * rows)
                + 0.4 * np.cos(11.0 * np.pi * cols) * np.sin(7.0 * np.pi * rows)
                + 0.25 * rng.standard_normal(shape))
    solution[0] = solution[-1] = 0.0
    solution[:, 0] = solution[:, -1] = 0.0
    return _five_point(solution), solution


def solver_scaling(sizes, methods=None, tolerance: float = 1e-8, max_iterations: int = 5000,
                   direct_limit: int = 600, seed: int = 0):
    """Time each method on square manufactured problems of the given sides."""
    methods = methods or ["direct", "cg", "multigrid", "mgcg"]
    results = {m: [] for m in methods}
    for size in sizes:
        b, solution = manufactured_problem((size, size), seed=seed)
        for method in methods:
            if method == "direct" and size > direct_limit:
                continue
            estimate, report = solve_system(b, method=method, tolerance=tolerance,
                                            max_iterations=max_iterations)
            results[method].append(BenchmarkRecord(
                method, (size, size), size * size, report.seconds, report.iterations,
                report.relative_residual, float(np.abs(estimate - solution).max())))
    return results


@dataclass
class BenchmarkTable:
    results: dict = field(default_factory=dict)

    def to_markdown(self) -> str:
        rows = sorted((r for recs in self.results.values() for r in recs),
                      key=lambda r: (r.unknowns, r.method))
        lines = ["| Grid | Unknowns | Method | Iterations | Seconds | Max error |",
                 "| --- | ---: | --- | ---: | ---: | ---: |"]
        for r in rows:
            its = "-" if r.iterations == 0 else str(r.iterations)
            lines.append(f"| {r.shape[0]} x {r.shape[1]} | {r.unknowns} | {r.method} | {its} | "
                         f"{r.seconds:.3f} | {r.max_error:.2e} |")
        return "\n".join(lines)
