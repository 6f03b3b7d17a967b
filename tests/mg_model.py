"""NumPy model of the B200 cell-centred V-cycle (test helper).

This restates, array by array, what the kernels of
``gradient_domain_b200/csrc/gd_mg_kernels.cuh`` compute, so that a single
V-cycle of the GPU plan (``PoissonPlan.apply_vcycle``) can be compared with it
to rounding level in FP64.  It is not the reference oracle (the reference has
no cell-centred multigrid); solution parity against the reference goes
through ``oracle``.
"""

from __future__ import annotations

import numpy as np

COARSEST_CELLS = 64


def rect_walls(shape):
    ny, nx = shape
    y = np.arange(ny)[:, None]
    x = np.arange(nx)[None, :]
    return ((y == 0).astype(int) + (y == ny - 1) + (x == 0) + (x == nx - 1))


def mask_classes(active):
    """0 for no unknown, else 1 + number of missing (inactive or outside) neighbours."""
    p = np.pad(active, 1)
    missing = (~p[:-2, 1:-1]).astype(int) + ~p[2:, 1:-1] + ~p[1:-1, :-2] + ~p[1:-1, 2:]
    return np.where(active, 1 + missing, 0)


class Level:
    def __init__(self, shape, boundary, level, active=None):
        self.shape = shape
        self.boundary = boundary
        self.wall = 0.0 if boundary == "neumann" else (1.0 if level == 0 else 2.0)
        if boundary == "masked":
            self.active = active
            self.cls = mask_classes(active)
        else:
            self.active = np.ones(shape, dtype=bool)
            self.cls = 1 + rect_walls(shape)
        walls = np.where(self.cls > 0, self.cls - 1, 0)
        self.diag = np.where(self.active, 4.0 - walls * (1.0 - self.wall), 1.0)
        yy, xx = np.mgrid[0:shape[0], 0:shape[1]]
        self.colour = (yy + xx) % 2

    def nbr(self, u):
        p = np.pad(u, 1)
        return p[:-2, 1:-1] + p[2:, 1:-1] + p[1:-1, :-2] + p[1:-1, 2:]

    def apply(self, u):
        return np.where(self.active, self.diag * u - self.nbr(u), 0.0)

    def sweep(self, u, b, colour):
        new = (b + self.nbr(u)) / self.diag
        return np.where(self.active & (self.colour == colour), new, u)


def build_levels(shape, boundary, active=None):
    levels = [Level(shape, boundary, 0, active)]
    while levels[-1].shape[0] * levels[-1].shape[1] > COARSEST_CELLS:
        ny, nx = levels[-1].shape
        cy, cx = (ny + 1) // 2, (nx + 1) // 2
        act = None
        if boundary == "masked":
            a = np.zeros((2 * cy, 2 * cx), dtype=bool)
            a[:ny, :nx] = levels[-1].active
            act = a[0::2, 0::2] | a[1::2, 0::2] | a[0::2, 1::2] | a[1::2, 1::2]
        levels.append(Level((cy, cx), boundary, len(levels), act))
    return levels


def prolong_1d(nf, nc, neumann):
    """Fine x coarse matrix: fine i takes 3/4 of coarse i//2 and 1/4 of its other neighbour."""
    p = np.zeros((nf, nc))
    for i in range(nf):
        c = i // 2
        c2 = c + 1 if i % 2 else c - 1
        p[i, c] += 0.75
        if 0 <= c2 < nc:
            p[i, c2] += 0.25
        elif neumann:
            p[i, min(max(c2, 0), nc - 1)] += 0.25
    return p


def coarse_inverse(L: Level):
    n = L.shape[0] * L.shape[1]
    a = np.zeros((n, n))
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        a[:, k] = L.apply(e.reshape(L.shape)).ravel()
    act = L.active.ravel()
    for k in np.nonzero(~act)[0]:
        a[k, :] = 0.0
        a[:, k] = 0.0
        a[k, k] = 1.0
    if L.boundary == "neumann":
        a += 1.0 / n
    return np.linalg.inv(a)


def vcycle(levels, b, sweeps=2, l=0):
    L = levels[l]
    if l == len(levels) - 1:
        return (coarse_inverse(L) @ b.ravel()).reshape(L.shape)
    u = np.zeros_like(b)
    for _ in range(sweeps):
        u = L.sweep(u, b, 0)
        u = L.sweep(u, b, 1)
    r = b - L.apply(u)
    neu = L.boundary == "neumann"
    C = levels[l + 1]
    pr = prolong_1d(L.shape[0], C.shape[0], neu)
    pc = prolong_1d(L.shape[1], C.shape[1], neu)
    bc = np.where(C.active, pr.T @ r @ pc, 0.0)
    e = vcycle(levels, bc, sweeps, l + 1)
    u = np.where(L.active, u + pr @ e @ pc.T, 0.0)
    for _ in range(sweeps):
        u = L.sweep(u, b, 1)
        u = L.sweep(u, b, 0)
    return u


def mgpcg(f, boundary, active=None, sweeps=2, tol=1e-8, max_it=200):
    """Plain FP64 PCG with the model V-cycle; returns (x, iterations)."""
    levels = build_levels(f.shape, boundary, active)
    A = levels[0]
    f = np.where(A.active, f, 0.0)
    if boundary == "neumann":
        f = f - f.mean()
    x = np.zeros_like(f)
    r = f.copy()
    ff = float(np.sum(f * f))
    p = np.zeros_like(f)
    rz_old = None
    for it in range(1, max_it + 1):
        z = vcycle(levels, r, sweeps)
        rz = float(np.sum(r * z))
        p = z if rz_old is None else z + (rz / rz_old) * p
        rz_old = rz
        q = A.apply(p)
        alpha = rz / float(np.sum(p * q))
        x += alpha * p
        r -= alpha * q
        if float(np.sum(r * r)) <= tol * tol * ff:
            return x, it
    return x, max_it
