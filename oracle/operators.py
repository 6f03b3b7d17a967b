"""Discrete operators of the reference, restated (oracle; test infrastructure).

Follows ``gradient-domain/src/gradient_domain/operators.py``.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def gradient(image):
    """Forward differences; last column of gx and last row of gy are zero.

    Follows gradient-domain/src/gradient_domain/operators.py:30-50.
    """
    image = np.asarray(image, dtype=float)
    gx = np.zeros(image.shape)
    gy = np.zeros(image.shape)
    gx[:, :-1] = np.diff(image, axis=1)
    gy[:-1, :] = np.diff(image, axis=0)
    return gx, gy


def divergence(gx, gy):
    """Negative adjoint of ``gradient`` (backward differences, edge terms).

    Follows gradient-domain/src/gradient_domain/operators.py:53-83.
    """
    gx = np.asarray(gx, dtype=float)
    gy = np.asarray(gy, dtype=float)
    out_x = np.zeros(gx.shape)
    out_y = np.zeros(gy.shape)
    if gx.shape[1] > 1:
        out_x[:, 0] = gx[:, 0]
        out_x[:, 1:-1] = gx[:, 1:-1] - gx[:, :-2]
        out_x[:, -1] = -gx[:, -2]
    if gy.shape[0] > 1:
        out_y[0] = gy[0]
        out_y[1:-1] = gy[1:-1] - gy[:-2]
        out_y[-1] = -gy[-2]
    return out_x + out_y


def neighbour_sum(u, mode="zero"):
    """Sum of the four neighbours in the reference's order (up, down, left, right)."""
    padded = np.pad(u, ((1, 1), (1, 1)) + ((0, 0),) * (u.ndim - 2),
                    mode="constant" if mode == "zero" else "edge")
    return padded[:-2, 1:-1] + padded[2:, 1:-1] + padded[1:-1, :-2] + padded[1:-1, 2:]


def laplacian(u, spacing=1.0):
    """Five-point Laplacian with zero outside the array, scaled by 1/h^2.

    Follows gradient-domain/src/gradient_domain/operators.py:86-107.
    """
    u = np.asarray(u, dtype=float)
    return (neighbour_sum(u) - 4.0 * u) / (spacing * spacing)


def neumann_laplacian(u):
    """``divergence(*gradient(u))``: edge-replicated five-point Laplacian.

    Equivalent form pinned by gradient-domain/tests/test_operators.py:51-57.
    """
    u = np.asarray(u, dtype=float)
    return neighbour_sum(u, mode="edge") - 4.0 * u


def sparse_laplacian(shape, spacing=1.0):
    """CSR assembly of ``laplacian`` (Kronecker sum of 1-D second differences).

    Follows gradient-domain/src/gradient_domain/operators.py:110-136.
    """
    def second_difference(size):
        return sp.diags([np.ones(size - 1), -2.0 * np.ones(size), np.ones(size - 1)],
                        [-1, 0, 1], format="csr")

    rows, cols = shape
    op = sp.kron(second_difference(rows), sp.identity(cols)) + sp.kron(
        sp.identity(rows), second_difference(cols))
    return (op / (spacing * spacing)).tocsr()


def fold_boundary(rhs, boundary, spacing=1.0):
    """Move the known Dirichlet ring of ``boundary`` into the interior RHS.

    Follows gradient-domain/src/gradient_domain/operators.py:139-169.
    """
    out = np.array(rhs, dtype=float, copy=True)
    w = 1.0 / (spacing * spacing)
    out[0] -= w * boundary[0, 1:-1]
    out[-1] -= w * boundary[-1, 1:-1]
    out[:, 0] -= w * boundary[1:-1, 0]
    out[:, -1] -= w * boundary[1:-1, -1]
    return out
