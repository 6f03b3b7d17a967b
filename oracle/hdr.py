"""The reference's gradient-domain tone mapping, restated (oracle).

Follows ``gradient-domain/src/gradient_domain/hdr.py``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .operators import divergence, gradient
from .solvers import solve_neumann

LUMA = np.array([0.2126, 0.7152, 0.0722])


@dataclass
class ToneMapConfig:
    """gradient-domain/src/gradient_domain/hdr.py:37-70."""

    alpha: float = 0.1
    beta: float = 0.85
    saturation: float = 0.5
    levels: int = 8
    epsilon: float = 1e-4


_BINOMIAL = np.array([1.0, 4.0, 6.0, 4.0, 1.0]) / 16.0


def downsample(image):
    """Separable binomial blur with edge padding, then decimate by 2,
    gradient-domain/src/gradient_domain/hdr.py:73-80."""
    w = image.shape[1]
    p = np.pad(image, ((0, 0), (2, 2)), mode="edge")
    blur = sum(k * p[:, i:i + w] for i, k in enumerate(_BINOMIAL))
    h = image.shape[0]
    p = np.pad(blur, ((2, 2), (0, 0)), mode="edge")
    blur = sum(k * p[i:i + h, :] for i, k in enumerate(_BINOMIAL))
    return blur[::2, ::2]


def upsample(image, shape):
    """Bilinear resampling on linspace grids, gradient-domain/src/gradient_domain/hdr.py:83-96."""
    ry = np.linspace(0, image.shape[0] - 1, shape[0])
    rx = np.linspace(0, image.shape[1] - 1, shape[1])
    y0, x0 = np.floor(ry).astype(int), np.floor(rx).astype(int)
    y1 = np.minimum(y0 + 1, image.shape[0] - 1)
    x1 = np.minimum(x0 + 1, image.shape[1] - 1)
    wy, wx = (ry - y0)[:, None], (rx - x0)[None, :]
    top = image[y0][:, x0] * (1 - wx) + image[y0][:, x1] * wx
    bot = image[y1][:, x0] * (1 - wx) + image[y1][:, x1] * wx
    return top * (1 - wy) + bot * wy


def central_gradient(image, spacing):
    """gradient-domain/src/gradient_domain/hdr.py:99-104."""
    p = np.pad(image, 1, mode="edge")
    return ((p[1:-1, 2:] - p[1:-1, :-2]) / (2.0 * spacing),
            (p[2:, 1:-1] - p[:-2, 1:-1]) / (2.0 * spacing))


def attenuation_field(log_lum, config):
    """Multiscale Fattal attenuation, gradient-domain/src/gradient_domain/hdr.py:107-134."""
    pyramid = [log_lum]
    while len(pyramid) < config.levels and min(pyramid[-1].shape) > 16:
        pyramid.append(downsample(pyramid[-1]))
    factor = None
    for level in reversed(range(len(pyramid))):
        gx, gy = central_gradient(pyramid[level], 2.0 ** level)
        mag = np.sqrt(gx * gx + gy * gy)
        scale = config.alpha * max(float(mag.mean()), config.epsilon)
        floor = np.maximum(mag, config.epsilon)
        local = (scale / floor) * (floor / scale) ** config.beta
        factor = local if factor is None else upsample(factor, local.shape) * local
    return factor


def tone_map(radiance, config=None):
    """gradient-domain/src/gradient_domain/hdr.py:137-185."""
    config = config or ToneMapConfig()
    radiance = np.asarray(radiance, dtype=float)
    if radiance.ndim != 3 or radiance.shape[2] != 3:
        raise ValueError("tone mapping expects a three-channel radiance map")
    lum = np.maximum(radiance @ LUMA, np.finfo(float).tiny)
    log_lum = np.log(lum)
    factor = attenuation_field(log_lum, config)
    gx, gy = gradient(log_lum)
    compressed = solve_neumann(divergence(gx * factor, gy * factor))
    result = np.exp(compressed - compressed.max())
    image = ((radiance / lum[..., None]) ** config.saturation) * result[..., None]
    peak = float(np.percentile(image, 99.5))
    return np.clip(image / max(peak, 1e-12), 0.0, 1.0), factor
