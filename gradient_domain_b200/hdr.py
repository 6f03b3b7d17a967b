"""Gradient-domain HDR tone mapping on the GPU Neumann solver.

Same interface as gradient-domain/src/gradient_domain/hdr.py: ``ToneMapConfig``
(:37-70), ``attenuation_field`` (:107-134) and ``tone_map`` (:137-185).  The
Poisson integration (the ``solve_neumann`` call at hdr.py:175) runs in the
B200 Neumann MGPCG; the attenuation pyramid and the final exposure/saturation
steps are the reference's array expressions, evaluated on the host.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .operators import divergence, gradient
from .solvers import solve_neumann

__all__ = ["ToneMapConfig", "attenuation_field", "tone_map"]

LUMA = np.array([0.2126, 0.7152, 0.0722])


@dataclass
class ToneMapConfig:
    """Attenuation parameters (hdr.py:37-70)."""

    alpha: float = 0.1
    beta: float = 0.85
    saturation: float = 0.5
    levels: int = 8
    epsilon: float = 1e-4


_BINOMIAL = np.array([1.0, 4.0, 6.0, 4.0, 1.0]) / 16.0


def _downsample(image: np.ndarray) -> np.ndarray:
    """Separable 5-tap binomial blur with edge replication, then keep every other sample."""
    width = image.shape[1]
    p = np.pad(image, ((0, 0), (2, 2)), mode="edge")
    blurred = sum(k * p[:, i:i + width] for i, k in enumerate(_BINOMIAL))
    height = image.shape[0]
    p = np.pad(blurred, ((2, 2), (0, 0)), mode="edge")
    blurred = sum(k * p[i:i + height, :] for i, k in enumerate(_BINOMIAL))
    return blurred[::2, ::2]


def _upsample(image: np.ndarray, shape) -> np.ndarray:
    """Bilinear resampling onto a finer grid spanning the same extent."""
    ry = np.linspace(0, image.shape[0] - 1, shape[0])
    rx = np.linspace(0, image.shape[1] - 1, shape[1])
    y0, x0 = np.floor(ry).astype(int), np.floor(rx).astype(int)
    y1 = np.minimum(y0 + 1, image.shape[0] - 1)
    x1 = np.minimum(x0 + 1, image.shape[1] - 1)
    wy, wx = (ry - y0)[:, None], (rx - x0)[None, :]
    top = image[y0][:, x0] * (1 - wx) + image[y0][:, x1] * wx
    bottom = image[y1][:, x0] * (1 - wx) + image[y1][:, x1] * wx
    return top * (1 - wy) + bottom * wy


def _central_gradient(image: np.ndarray, spacing: float):
    p = np.pad(image, 1, mode="edge")
    return ((p[1:-1, 2:] - p[1:-1, :-2]) / (2.0 * spacing),
            (p[2:, 1:-1] - p[:-2, 1:-1]) / (2.0 * spacing))


def attenuation_field(log_luminance, config: ToneMapConfig) -> np.ndarray:
    """Multiscale gradient attenuation factor, propagated coarse to fine."""
    pyramid = [np.asarray(log_luminance, dtype=float)]
    while len(pyramid) < config.levels and min(pyramid[-1].shape) > 16:
        pyramid.append(_downsample(pyramid[-1]))
    factor = None
    for level in reversed(range(len(pyramid))):
        gx, gy = _central_gradient(pyramid[level], 2.0 ** level)
        magnitude = np.sqrt(gx * gx + gy * gy)
        scale = config.alpha * max(float(magnitude.mean()), config.epsilon)
        floored = np.maximum(magnitude, config.epsilon)
        local = (scale / floored) * (floored / scale) ** config.beta
        factor = local if factor is None else _upsample(factor, local.shape) * local
    return factor


def tone_map(radiance, config: ToneMapConfig | None = None):
    """Compress a linear HDR radiance map (h, w, 3) to display values in [0, 1].

    Raises ``ValueError`` if the input is not a three-channel image.
    """
    config = config or ToneMapConfig()
    radiance = np.asarray(radiance, dtype=float)
    if radiance.ndim != 3 or radiance.shape[2] != 3:
        raise ValueError("tone mapping expects a three-channel radiance map")
    luminance = np.maximum(radiance @ LUMA, np.finfo(float).tiny)
    log_luminance = np.log(luminance)
    factor = attenuation_field(log_luminance, config)
    gx, gy = gradient(log_luminance)
    compressed = solve_neumann(divergence(gx * factor, gy * factor))
    result = np.exp(compressed - compressed.max())
    image = ((radiance / luminance[..., None]) ** config.saturation) * result[..., None]
    peak = float(np.percentile(image, 99.5))
    return np.clip(image / max(peak, 1e-12), 0.0, 1.0), factor
