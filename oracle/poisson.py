"""The reference's Poisson editing entry points, restated (oracle).

Follows ``gradient-domain/src/gradient_domain/poisson.py``.
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .operators import divergence, fold_boundary, gradient
from .solvers import SolverReport, solve_system


@dataclass
class GuidanceField:
    """gradient-domain/src/gradient_domain/poisson.py:52-92."""

    gx: np.ndarray
    gy: np.ndarray

    @classmethod
    def of(cls, image):
        return cls(*gradient(image))

    def select(self, mask, other):
        sel = mask[..., None] if self.gx.ndim == 3 else mask
        return GuidanceField(np.where(sel, self.gx, other.gx), np.where(sel, self.gy, other.gy))

    def mix_by_magnitude(self, other):
        return GuidanceField(np.where(np.abs(self.gx) >= np.abs(other.gx), self.gx, other.gx),
                             np.where(np.abs(self.gy) >= np.abs(other.gy), self.gy, other.gy))

    def scaled(self, factor):
        return GuidanceField(self.gx * factor, self.gy * factor)


def solve_dirichlet(field, boundary, method="mgcg", tolerance=1e-8, max_iterations=2000):
    """Per-channel rectangle solve, gradient-domain/src/gradient_domain/poisson.py:102-147."""
    bnd = np.asarray(boundary, dtype=float)
    gray = bnd.ndim == 2
    chans = bnd[..., None] if gray else bnd
    rhs = divergence(field.gx, field.gy)
    if rhs.ndim == 2:
        rhs = rhs[..., None]
    out = chans.copy()
    reports = []
    for c in range(chans.shape[2]):
        folded = fold_boundary(rhs[1:-1, 1:-1, c], chans[..., c])
        sol, rep = solve_system(folded, method=method, tolerance=tolerance,
                                max_iterations=max_iterations)
        out[1:-1, 1:-1, c] = sol
        reports.append(rep)
    return (out[..., 0] if gray else out), reports


_OFFSETS = ((-1, 0), (1, 0), (0, -1), (0, 1))


def masked_system(mask):
    """Unknown numbering and CSR operator of the masked problem,
    gradient-domain/src/gradient_domain/poisson.py:180-204."""
    interior = np.zeros_like(mask, dtype=bool)
    interior[1:-1, 1:-1] = mask[1:-1, 1:-1]
    n = int(interior.sum())
    index = np.full(mask.shape, -1, dtype=np.int64)
    index[interior] = np.arange(n)
    rows, cols, vals = [np.arange(n)], [np.arange(n)], [np.full(n, -4.0)]
    for dr, dc in _OFFSETS:
        nb = np.roll(np.roll(index, -dr, axis=0), -dc, axis=1)[interior]
        ok = nb >= 0
        rows.append(np.arange(n)[ok])
        cols.append(nb[ok])
        vals.append(np.ones(int(ok.sum())))
    op = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                       shape=(n, n))
    return interior, index, op


def masked_rhs(rhs_channel, values, interior, index):
    """Divergence minus out-of-mask neighbour values,
    gradient-domain/src/gradient_domain/poisson.py:216-224."""
    b = rhs_channel[interior].astype(float)
    for dr, dc in _OFFSETS:
        nb_index = np.roll(np.roll(index, -dr, axis=0), -dc, axis=1)[interior]
        nb_value = np.roll(np.roll(values, -dr, axis=0), -dc, axis=1)[interior]
        outside = nb_index < 0
        b[outside] -= nb_value[outside]
    return b


def solve_masked(field, image, mask):
    """Masked Perez solve by SuperLU, gradient-domain/src/gradient_domain/poisson.py:154-244."""
    img = np.asarray(image, dtype=float)
    gray = img.ndim == 2
    chans = img[..., None] if gray else img
    interior, index, op = masked_system(mask)
    if not interior.any():
        return img.copy(), []
    t0 = time.perf_counter()
    lu = spla.splu(op.tocsc())
    t_fact = time.perf_counter() - t0
    rhs = divergence(field.gx, field.gy)
    if rhs.ndim == 2:
        rhs = rhs[..., None]
    out = chans.copy()
    reports = []
    for c in range(chans.shape[2]):
        b = masked_rhs(rhs[..., c], chans[..., c], interior, index)
        t0 = time.perf_counter()
        x = lu.solve(b)
        dt = time.perf_counter() - t0
        out[..., c][interior] = x
        res = float(np.linalg.norm(op @ x - b)) / max(float(np.linalg.norm(b)), 1e-30)
        reports.append(SolverReport("direct (masked)", 0, res, dt + t_fact / chans.shape[2], True))
    return (out[..., 0] if gray else out), reports


def place(source, mask, target_shape, offset):
    """gradient-domain/src/gradient_domain/poisson.py:247-258."""
    r, c = offset
    h, w = source.shape[:2]
    if r < 0 or c < 0 or r + h > target_shape[0] or c + w > target_shape[1]:
        raise ValueError("source patch does not fit the target at this offset")
    canvas = np.zeros(target_shape)
    canvas[r:r + h, c:c + w] = source
    placed = np.zeros(target_shape[:2], dtype=bool)
    placed[r:r + h, c:c + w] = mask
    return canvas, placed


def clone_field(source, target, mask, offset, mode):
    """Guidance field of seamless_clone, gradient-domain/src/gradient_domain/poisson.py:310-330."""
    target = np.asarray(target, dtype=float)
    source = np.asarray(source, dtype=float)
    if source.ndim != target.ndim:
        raise ValueError("source and target must have the same number of dimensions")
    canvas, placed = place(source, mask, target.shape, offset)
    fs, ft = GuidanceField.of(canvas), GuidanceField.of(target)
    if mode == "import":
        inside = fs
    elif mode == "mixed":
        inside = fs.mix_by_magnitude(ft)
    elif mode == "average":
        inside = GuidanceField(0.5 * (fs.gx + ft.gx), 0.5 * (fs.gy + ft.gy))
    else:
        raise ValueError(f"unknown mode {mode!r}")
    return inside.select(placed, ft), placed, target


def seamless_clone(source, target, mask, offset=(0, 0), mode="import", domain="mask",
                   method="mgcg", margin=24):
    """gradient-domain/src/gradient_domain/poisson.py:261-348."""
    field, placed, target = clone_field(source, target, mask, offset, mode)
    if domain == "mask":
        return solve_masked(field, target, placed)
    if domain != "rectangle":
        raise ValueError(f"unknown domain {domain!r}")
    rows, cols = np.nonzero(placed)
    top, bottom = max(int(rows.min()) - margin, 0), min(int(rows.max()) + margin + 1, target.shape[0])
    left, right = max(int(cols.min()) - margin, 0), min(int(cols.max()) + margin + 1, target.shape[1])
    win = (slice(top, bottom), slice(left, right))
    patch, reports = solve_dirichlet(GuidanceField(field.gx[win], field.gy[win]), target[win],
                                     method=method)
    out = target.copy()
    out[win] = patch
    return out, reports


def texture_flatten(image, edges, method="mgcg", mask=None):
    """gradient-domain/src/gradient_domain/poisson.py:351-388."""
    image = np.asarray(image, dtype=float)
    w = np.asarray(edges, dtype=float)
    if image.ndim == 3:
        w = w[..., None]
    field = GuidanceField.of(image).scaled(w)
    if mask is not None:
        return solve_masked(field, image, mask)
    return solve_dirichlet(field, image, method=method)


def illumination_change(image, mask, alpha=0.2, beta=0.2, epsilon=1e-4):
    """gradient-domain/src/gradient_domain/poisson.py:391-431."""
    image = np.asarray(image, dtype=float)
    f = GuidanceField.of(image)
    mag = np.sqrt(f.gx ** 2 + f.gy ** 2)
    factor = (alpha ** beta) * np.maximum(mag, epsilon) ** (-beta)
    return solve_masked(f.scaled(factor), image, mask)
