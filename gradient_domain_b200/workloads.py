"""Seeded synthetic inputs for the benchmark configurations of this path.

Every generator runs on the host in FP64 with ``numpy.random.default_rng`` so
the GPU solver and the CPU baseline see identical inputs.

* ``neumann_blobs``: a single-channel integration problem, the forward
  gradient field of a sum of 32 isotropic Gaussian blobs (centres uniform,
  sigma uniform in [10, 120] px, amplitude uniform in [0, 1]) plus uniform
  noise of amplitude 0.05, with Neumann boundaries (1024 x 1024 by default).
* ``tonemap_rhs``: a tone-mapping-style three-channel problem: per channel a
  log-normal radiance (log-mean 0, log-std 2.5) modulated by 64 Gaussian
  blobs; the guidance field is the forward gradient of the log radiance
  attenuated by the multiscale factor with alpha = 0.1 * mean |g|,
  beta = 0.85 and one pyramid level (hdr.py:107-134); Neumann boundaries
  (4096 x 4096 x 3 by default).
* ``composite_case``: seamless compositing of two blob images inside a
  random 12-vertex star polygon (radii 300-800 px around the centre of a
  2048 x 2048 canvas), the reference's masked setup (poisson.py:154-244).
"""

from __future__ import annotations

import numpy as np

from .hdr import ToneMapConfig, attenuation_field


def blob_image(shape, count, rng, sigma=(10.0, 120.0), noise=0.05):
    """Sum of isotropic Gaussian blobs plus uniform noise, via one GEMM."""
    h, w = shape
    cy = rng.uniform(0, h, count)
    cx = rng.uniform(0, w, count)
    s = rng.uniform(sigma[0], sigma[1], count)
    a = rng.uniform(0.0, 1.0, count)
    ys = np.exp(-((np.arange(h)[:, None] - cy[None, :]) ** 2) / (2 * s * s))
    xs = np.exp(-((np.arange(w)[:, None] - cx[None, :]) ** 2) / (2 * s * s))
    img = (ys * a[None, :]) @ xs.T
    if noise:
        img += noise * rng.random(shape)
    return img


def forward_gradient(u):
    gx = np.zeros_like(u)
    gy = np.zeros_like(u)
    gx[:, :-1] = u[:, 1:] - u[:, :-1]
    gy[:-1, :] = u[1:, :] - u[:-1, :]
    return gx, gy


def divergence(gx, gy):
    out = np.zeros_like(gx)
    out[:, 0] += gx[:, 0]
    out[:, 1:-1] += gx[:, 1:-1] - gx[:, :-2]
    out[:, -1] -= gx[:, -2]
    out[0, :] += gy[0, :]
    out[1:-1, :] += gy[1:-1, :] - gy[:-2, :]
    out[-1, :] -= gy[-2, :]
    return out


def neumann_blobs(size=1024, seed=0):
    """(rhs, source): rhs = divergence(gradient(source)), the Neumann Laplacian."""
    rng = np.random.default_rng(seed)
    src = blob_image((size, size), 32, rng)
    return divergence(*forward_gradient(src)), src


def tonemap_rhs(size=4096, seed=1, channels=3):
    """Per-channel Neumann right-hand sides (channels, size, size) of the tone-mapping case."""
    rng = np.random.default_rng(seed)
    scale = size / 1024.0
    out = np.empty((channels, size, size))
    cfg = ToneMapConfig(alpha=0.1, beta=0.85, levels=1)
    for c in range(channels):
        mod = 0.05 + blob_image((size, size), 64, rng, sigma=(10.0 * scale, 120.0 * scale),
                                noise=0.0)
        log_r = 2.5 * rng.standard_normal((size, size)) + np.log(mod)
        factor = attenuation_field(log_r, cfg)
        gx, gy = forward_gradient(log_r)
        out[c] = divergence(gx * factor, gy * factor)
    return out


def star_polygon_mask(size, rng, vertices=12, rmin=300.0, rmax=800.0):
    """Even-odd rasterisation at pixel centres of a random star polygon."""
    ang = 2 * np.pi * np.arange(vertices) / vertices + rng.uniform(-0.2, 0.2, vertices)
    rad = rng.uniform(rmin, rmax, vertices)
    c = size / 2.0
    vy, vx = c + rad * np.sin(ang), c + rad * np.cos(ang)
    yy = np.arange(size)[:, None] + 0.5
    xx = np.arange(size)[None, :] + 0.5
    inside = np.zeros((size, size), dtype=bool)
    j = vertices - 1
    for i in range(vertices):
        crosses = (vy[i] > yy) != (vy[j] > yy)
        with np.errstate(divide="ignore", invalid="ignore"):
            xint = (vx[j] - vx[i]) * (yy - vy[i]) / (vy[j] - vy[i]) + vx[i]
        inside ^= crosses & (xx < xint)
        j = i
    return inside


def composite_case(size=2048, seed=2):
    """(source, target, mask) images in [0, 1] and the star polygon selection."""
    rng = np.random.default_rng(seed)
    scale = size / 2048.0

    def image():
        img = np.stack([blob_image((size, size), 32, rng, sigma=(10 * scale, 120 * scale))
                        for _ in range(3)], axis=2)
        img -= img.min()
        return img / max(img.max(), 1e-12)

    source, target = image(), image()
    mask = star_polygon_mask(size, rng, rmin=300 * scale, rmax=800 * scale)
    return source, target, mask
