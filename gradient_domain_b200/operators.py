"""Discrete operators on the GPU (gradient-domain/src/gradient_domain/operators.py).

``gradient`` (:30-50), ``divergence`` (:53-83), ``laplacian`` (:86-107) and
``fold_boundary`` (:139-169) run in the library's FP64 kernels with the
reference's order of operations; ``sparse_laplacian`` (:110-136) assembles the
same SciPy matrix on the host, because it builds a host data structure for
callers that want one and is not used by any solver here.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib
from ._host import download, upload

__all__ = ["gradient", "divergence", "laplacian", "sparse_laplacian", "fold_boundary"]


def _dev(a, dev) -> torch.Tensor:
    return upload(a, dev, np.float64)


def _channels_first(a: torch.Tensor) -> torch.Tensor:
    return a.unsqueeze(0) if a.dim() == 2 else a.permute(2, 0, 1).contiguous()


def _channels_last(a: torch.Tensor, ndim: int) -> np.ndarray:
    return download(a[0] if ndim == 2 else a.permute(1, 2, 0))


def gradient_dev(u: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """Forward differences of a (c, h, w) device tensor."""
    gx, gy = torch.empty_like(u), torch.empty_like(u)
    c, h, w = u.shape
    for k in range(c):
        _lib.check(_lib.lib().gd_gradient(_lib.ptr(gx[k]), _lib.ptr(gy[k]), _lib.ptr(u[k]), h, w,
                                          _lib.stream_handle()), "gd_gradient")
    return gx, gy


def divergence_dev(gx: torch.Tensor, gy: torch.Tensor) -> torch.Tensor:
    """Negative adjoint of the gradient for (c, h, w) device tensors."""
    out = torch.empty_like(gx)
    c, h, w = gx.shape
    for k in range(c):
        _lib.check(_lib.lib().gd_divergence(_lib.ptr(out[k]), _lib.ptr(gx[k]), _lib.ptr(gy[k]),
                                            h, w, _lib.stream_handle()), "gd_divergence")
    return out


def gradient(image) -> tuple[np.ndarray, np.ndarray]:
    """Forward differences; last column of gx and last row of gy are zero."""
    image = np.asarray(image, dtype=float)
    u = _channels_first(_dev(image, _lib.device()))
    gx, gy = gradient_dev(u)
    return _channels_last(gx, image.ndim), _channels_last(gy, image.ndim)


def divergence(gx, gy) -> np.ndarray:
    """Negative adjoint of :func:`gradient` (backward differences)."""
    gx = np.asarray(gx, dtype=float)
    dev = _lib.device()
    out = divergence_dev(_channels_first(_dev(gx, dev)), _channels_first(_dev(gy, dev)))
    return _channels_last(out, gx.ndim)


def laplacian(u, spacing: float = 1.0) -> np.ndarray:
    """Five-point Laplacian with zero outside the array, scaled by 1 / h^2."""
    u = np.asarray(u, dtype=float)
    dev = _lib.device()
    ud = _channels_first(_dev(u, dev))
    zero = torch.zeros_like(ud[0])
    out = torch.empty_like(ud)
    c, m, n = ud.shape
    for k in range(c):
        # gd_ref_residual gives 0 - laplacian(u); negation is exact
        _lib.check(_lib.lib().gd_ref_residual(_lib.ptr(out[k]), _lib.ptr(ud[k]), _lib.ptr(zero),
                                              m, n, float(spacing), _lib.stream_handle()),
                   "gd_ref_residual")
    return -_channels_last(out, u.ndim)


def sparse_laplacian(shape, spacing: float = 1.0) -> sp.csr_matrix:
    """CSR matrix of :func:`laplacian` on an ``(m, n)`` grid, row-major."""
    rows, cols = shape

    def second_difference(size):
        return sp.diags([np.ones(size - 1), np.full(size, -2.0), np.ones(size - 1)], [-1, 0, 1],
                        format="csr")

    op = sp.kron(second_difference(rows), sp.identity(cols, format="csr")) + sp.kron(
        sp.identity(rows, format="csr"), second_difference(cols))
    return (op / (spacing * spacing)).tocsr()


def fold_boundary(right_hand_side, boundary, spacing: float = 1.0) -> np.ndarray:
    """Move the Dirichlet ring of ``boundary`` into the interior right-hand side."""
    rhs = np.asarray(right_hand_side, dtype=float)
    bnd = np.asarray(boundary, dtype=float)
    if rhs.ndim not in (2, 3) or bnd.ndim != rhs.ndim:
        raise ValueError("right_hand_side and boundary must both be (h, w) or (h, w, c)")
    h, w = bnd.shape[:2]
    channels = bnd.shape[2] if bnd.ndim == 3 else 1
    if rhs.shape != (h - 2, w - 2) + bnd.shape[2:]:
        raise ValueError(f"right_hand_side {rhs.shape} is not the interior of boundary {bnd.shape}")
    dev = _lib.device()
    rd = _dev(rhs, dev)
    out = torch.empty_like(rd)
    _lib.check(_lib.lib().gd_fold_boundary(_lib.ptr(out), _lib.ptr(rd), _lib.ptr(_dev(bnd, dev)),
                                           h, w, channels, float(spacing), _lib.stream_handle()),
               "gd_fold_boundary")
    return download(out)
