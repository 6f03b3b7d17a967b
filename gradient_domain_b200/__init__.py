"""B200-native gradient-domain Poisson integration.

Drop-in replacement for the Poisson path of the ``gradient_domain`` package
(Giankaqui/visual-computing, ``gradient-domain/src/gradient_domain``): the same
solver entry points, report types and argument conventions, with every solve
running in hand-written sm_100a CUDA kernels behind the C ABI of
``include/gd_poisson.h``.
"""

from .benchmark import BenchmarkRecord, BenchmarkTable, manufactured_problem, solver_scaling
from .hdr import ToneMapConfig, attenuation_field, tone_map
from .multigrid import MultigridOptions, MultigridReport, smooth, solve, v_cycle
from .operators import divergence, fold_boundary, gradient, laplacian, sparse_laplacian
from .plan import Instance, PoissonPlan, SolveParams, cached_plan
from .poisson import (
    GuidanceField,
    illumination_change,
    seamless_clone,
    solve_dirichlet,
    solve_masked,
    texture_flatten,
)
from .solvers import (SOLVERS, NeumannBatchFuture, SolverReport, solve_neumann,
                      solve_neumann_batch, solve_neumann_batch_async, solve_system)

__all__ = [
    "SOLVERS", "BenchmarkRecord", "BenchmarkTable", "GuidanceField", "Instance",
    "MultigridOptions", "MultigridReport", "NeumannBatchFuture", "PoissonPlan", "SolveParams",
    "SolverReport",
    "ToneMapConfig", "attenuation_field", "cached_plan", "divergence", "fold_boundary",
    "gradient", "illumination_change", "laplacian", "manufactured_problem", "seamless_clone",
    "solve", "solve_dirichlet", "solve_masked", "solve_neumann", "solve_neumann_batch",
    "solve_neumann_batch_async", "solve_system",
    "smooth", "solver_scaling", "sparse_laplacian", "texture_flatten", "tone_map", "v_cycle",
]

__version__ = "0.1.0"
