"""Reference-exact geometric multigrid on the GPU.

Same interface and semantics as gradient-domain/src/gradient_domain/multigrid.py:
``MultigridOptions`` (:47-71), ``MultigridReport`` (:75-108), ``v_cycle``
(:184-215) and ``solve`` (:218-255).  The V-cycle runs in the library's
vertex-centred FP64 kernels (``gd_ref_vcycle``), which evaluate every
smoothing, residual and transfer expression in the reference's order, so one
cycle matches the NumPy one to rounding and ``solve`` takes the same number of
cycles.  The B200 solver proper (cell-centred, mixed precision, batched) is
``gradient_domain_b200.solvers`` method ``"mgcg"``.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._host import download, upload


@dataclass
class MultigridOptions:
    """Smoother and recursion settings (multigrid.py:47-71)."""

    pre_smoothing: int = 2
    post_smoothing: int = 2
    coarsest_size: int = 8
    coarsest_sweeps: int = 60
    max_cycles: int = 60
    tolerance: float = 1e-8


@dataclass
class MultigridReport:
    """Convergence record of one solve (multigrid.py:75-108)."""

    residuals: list = field(default_factory=list)
    cycles: int = 0
    converged: bool = False

    @property
    def convergence_factor(self) -> float:
        if len(self.residuals) < 2 or self.residuals[0] <= 0:
            return float("nan")
        ratio = self.residuals[-1] / self.residuals[0]
        return float(ratio ** (1.0 / (len(self.residuals) - 1)))

    def __str__(self) -> str:
        return (f"{self.cycles} cycles, relative residual {self.residuals[-1]:.2e}, "
                f"convergence factor {self.convergence_factor:.3f}")


class RefWorkspace:
    """Device scratch of the reference-exact kernels for one grid shape."""

    def __init__(self, shape: tuple[int, int], coarsest_size: int, dev: torch.device):
        m, n = shape
        nbytes = int(_lib.lib().gd_ref_workspace_bytes(m, n, coarsest_size))
        if nbytes == 0:
            raise ValueError(f"unsupported grid {shape}")
        self.buf = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        self.dot_buf = torch.empty(1024, dtype=torch.float64, device=dev)
        self.scalar = torch.empty(1, dtype=torch.float64, device=dev)
        self.shape, self.coarsest_size = shape, coarsest_size

    def vcycle(self, u: torch.Tensor, b: torch.Tensor, spacing: float, o: MultigridOptions):
        m, n = self.shape
        _lib.check(_lib.lib().gd_ref_vcycle(_lib.ptr(u), _lib.ptr(b), m, n, float(spacing),
                                            o.pre_smoothing, o.post_smoothing, o.coarsest_size,
                                            o.coarsest_sweeps, _lib.ptr(self.buf),
                                            self.buf.numel(), _lib.stream_handle()),
                   "gd_ref_vcycle")

    def residual(self, r: torch.Tensor, u: torch.Tensor, b: torch.Tensor, spacing: float):
        m, n = self.shape
        _lib.check(_lib.lib().gd_ref_residual(_lib.ptr(r), _lib.ptr(u), _lib.ptr(b), m, n,
                                              float(spacing), _lib.stream_handle()),
                   "gd_ref_residual")

    def dot(self, a: torch.Tensor, b: torch.Tensor) -> float:
        _lib.check(_lib.lib().gd_ref_dot(_lib.ptr(self.scalar), _lib.ptr(a), _lib.ptr(b),
                                         a.numel(), _lib.ptr(self.dot_buf),
                                         self.dot_buf.numel() * 8, _lib.stream_handle()),
                   "gd_ref_dot")
        return float(self.scalar.item())

    def axpby(self, y: torch.Tensor, x: torch.Tensor, alpha: float, beta: float) -> None:
        _lib.check(_lib.lib().gd_ref_axpby(_lib.ptr(y), _lib.ptr(x), float(alpha), float(beta),
                                           y.numel(), _lib.stream_handle()), "gd_ref_axpby")


def _to_dev(a, dev) -> torch.Tensor:
    return upload(a, dev, np.float64)


def smooth(u, b, spacing: float = 1.0, sweeps: int = 1):
    """``sweeps`` red-black Gauss-Seidel sweeps on ``laplacian(u) = b`` (multigrid.py:147-165).

    Returns a new array (NumPy in, NumPy out; a CUDA tensor in, a CUDA tensor
    out); ``u`` is not changed.  float64 gives the reference's ``_smooth``
    bitwise; when ``u`` and ``b`` are both float32 the sweeps run in float32,
    bitwise the same expression evaluated in float32.  Each device pass
    (``gd_rbgs_smooth``) runs up to four sweeps, reading u and b once.
    """
    dev = _lib.device()
    as_tensor = isinstance(u, torch.Tensor)
    fp32 = all((x.dtype == torch.float32) if isinstance(x, torch.Tensor)
               else (np.asarray(x).dtype == np.float32) for x in (u, b))
    dtype = torch.float32 if fp32 else torch.float64

    def to_dev(x):
        if isinstance(x, torch.Tensor):
            return x.to(device=dev, dtype=dtype).contiguous()
        return upload(np.asarray(x), dev, np.float32 if fp32 else np.float64)

    u_d, b_d = to_dev(u), to_dev(b)
    if u_d.dim() != 2 or u_d.shape != b_d.shape:
        raise ValueError("u and b must be 2-D arrays of the same shape")
    ny, nx = u_d.shape
    if sweeps <= 0 or u_d.numel() == 0:
        out = u_d.clone()
    else:
        out, spare = torch.empty_like(u_d), torch.empty_like(u_d)
        src, left = u_d, int(sweeps)
        while left > 0:
            k = min(4, left)
            dst = out if src is not out else spare
            _lib.check(_lib.lib().gd_rbgs_smooth(_lib.ptr(src), _lib.ptr(dst), _lib.ptr(b_d), ny,
                                                 nx, nx, 0 if fp32 else 1, float(spacing), k,
                                                 _lib.stream_handle()), "gd_rbgs_smooth")
            src, left = dst, left - k
        out = src
    return out if as_tensor else download(out)


def _restrict(residual) -> np.ndarray:
    """Full-weighting restriction, 0.25 Rows^T r Cols (multigrid.py:169-174), on the device;
    an (m, n) grid goes to ((m - 1) // 2, (n - 1) // 2)."""
    dev = _lib.device()
    r = _to_dev(np.asarray(residual, dtype=float), dev)
    m, n = r.shape
    rc = torch.empty(((m - 1) // 2, (n - 1) // 2), dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().gd_ref_restrict(_lib.ptr(rc), _lib.ptr(r), m, n, _lib.stream_handle()),
               "gd_ref_restrict")
    return download(rc)


def _prolong(correction, shape) -> np.ndarray:
    """Bilinear interpolation Rows e Cols^T of a coarse correction onto an ``shape`` grid,
    zero outside the coarse grid (multigrid.py:177-181), on the device."""
    dev = _lib.device()
    e = _to_dev(np.asarray(correction, dtype=float), dev)
    m, n = int(shape[0]), int(shape[1])
    u = torch.zeros((m, n), dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().gd_ref_prolong_add(_lib.ptr(u), _lib.ptr(e), m, n, e.shape[0],
                                             e.shape[1], _lib.stream_handle()),
               "gd_ref_prolong_add")
    return download(u)


def v_cycle(u, b, spacing: float, options: MultigridOptions) -> np.ndarray:
    """One V-cycle on ``laplacian(u) = b`` (multigrid.py:184-215); returns a new array."""
    dev = _lib.device()
    b_d = _to_dev(b, dev)
    u_d = _to_dev(u, dev).clone()
    if u_d.shape != b_d.shape or u_d.dim() != 2:
        raise ValueError("u and b must be 2-D arrays of the same shape")
    RefWorkspace(tuple(b_d.shape), options.coarsest_size, dev).vcycle(u_d, b_d, spacing, options)
    return download(u_d)


def solve(b, spacing: float = 1.0, options: MultigridOptions | None = None,
          initial=None) -> tuple[np.ndarray, MultigridReport]:
    """Repeated V-cycles until the relative residual is below tolerance (multigrid.py:218-255)."""
    options = options or MultigridOptions()
    b = np.asarray(b, dtype=float)
    dev = _lib.device()
    b_d = _to_dev(b, dev)
    u_d = torch.zeros_like(b_d) if initial is None else _to_dev(initial, dev).clone()
    ws = RefWorkspace(tuple(b_d.shape), options.coarsest_size, dev)
    scale = float(np.sqrt(ws.dot(b_d, b_d)))
    if scale == 0.0:
        return download(u_d), MultigridReport([0.0], 0, True)
    r_d = torch.empty_like(b_d)

    def rel_residual() -> float:
        ws.residual(r_d, u_d, b_d, spacing)
        return float(np.sqrt(ws.dot(r_d, r_d))) / scale

    history = [rel_residual()]
    for cycle in range(1, options.max_cycles + 1):
        ws.vcycle(u_d, b_d, spacing, options)
        history.append(rel_residual())
        if history[-1] < options.tolerance:
            return download(u_d), MultigridReport(history, cycle, True)
    return download(u_d), MultigridReport(history, options.max_cycles, False)
