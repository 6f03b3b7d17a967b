"""Gradient-domain HDR tone mapping on the GPU.

Same interface as gradient-domain/src/gradient_domain/hdr.py: ``ToneMapConfig``
(:37-70), ``attenuation_field`` (:107-134) and ``tone_map`` (:137-185).
``tone_map`` runs on the device from the uploaded radiance to the display
image: log-luminance, the attenuation pyramid (binomial downsampling, central
gradients, per-level factors propagated coarse to fine), the attenuated field
and its divergence, the Neumann solve (the reference's exact DCT algorithm,
gd_dct.cu), and the exposure / saturation / percentile normalisation
(gd_tonemap.cu, gd_rhs.cu); only the image and the factor come back.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._host import download, upload
from .plan import Instance, SolveParams, cached_plan

__all__ = ["ToneMapConfig", "attenuation_field", "tone_map"]

LUMA = np.array([0.2126, 0.7152, 0.0722])
NEUMANN_TOLERANCE = 1e-14  # the exact-solver level of solve_neumann


@dataclass
class ToneMapConfig:
    """Attenuation parameters (hdr.py:37-70)."""

    alpha: float = 0.1
    beta: float = 0.85
    saturation: float = 0.5
    levels: int = 8
    epsilon: float = 1e-4


def _scratch(dev) -> torch.Tensor:
    return torch.empty(int(_lib.lib().gd_tm_scratch_bytes()), dtype=torch.uint8, device=dev)


def _attenuation_dev(logl: torch.Tensor, config: ToneMapConfig,
                     scratch: torch.Tensor) -> torch.Tensor:
    """The multiscale attenuation factor of a device log-luminance (h, w)."""
    lib, st = _lib.lib(), _lib.stream_handle()
    pyramid = [logl]
    while len(pyramid) < config.levels and min(pyramid[-1].shape) > 16:
        h, w = pyramid[-1].shape
        out = torch.empty(((h + 1) // 2, (w + 1) // 2), dtype=torch.float64, device=logl.device)
        _lib.check(lib.gd_tm_downsample(_lib.ptr(out), _lib.ptr(pyramid[-1]), h, w, st),
                   "gd_tm_downsample")
        pyramid.append(out)
    factor = None
    for level in reversed(range(len(pyramid))):
        a = pyramid[level]
        h, w = a.shape
        f = torch.empty_like(a)
        ch, cw = factor.shape if factor is not None else (0, 0)
        _lib.check(lib.gd_tm_level_factor(_lib.ptr(f), _lib.ptr(a),
                                          _lib.ptr(factor) if factor is not None else None,
                                          h, w, ch, cw, 2.0 ** level, float(config.alpha),
                                          float(config.beta), float(config.epsilon),
                                          _lib.ptr(scratch), st), "gd_tm_level_factor")
        factor = f
    return factor


def attenuation_field(log_luminance, config: ToneMapConfig) -> np.ndarray:
    """Multiscale gradient attenuation factor, propagated coarse to fine."""
    dev = _lib.device()
    logl = upload(log_luminance, dev, np.float64)
    return download(_attenuation_dev(logl, config, _scratch(dev)))


def tone_map_device(rad: torch.Tensor, config: ToneMapConfig, dct=None):
    """The tone-mapping pipeline on a device radiance map (h, w, 3) FP64, on the
    current stream; returns the display image (h, w, 3) and the factor (h, w),
    both on the device.  ``dct`` is the DCT solver of this shape to use (a
    ``DctPlan``; by default the process-wide one of the shape)."""
    h, w, _ = rad.shape
    dev = rad.device
    lib, st = _lib.lib(), _lib.stream_handle()
    logl = torch.empty((h, w), dtype=torch.float64, device=dev)
    lum = torch.empty_like(logl)
    _lib.check(lib.gd_tm_log_luminance(_lib.ptr(logl), _lib.ptr(lum), _lib.ptr(rad), h, w, st),
               "gd_tm_log_luminance")
    scratch = _scratch(dev)
    factor = _attenuation_dev(logl, config, scratch)
    # forward-difference field of the log-luminance times the factor, and its
    # divergence over the whole image (hdr.py:171-175)
    div = torch.empty_like(logl)
    desc = _lib.FieldDesc(_lib.GD_FIELD_WEIGHTED, h, w, 1, 0, 1, _lib.ptr(logl), None, None,
                          _lib.ptr(factor), 0.0, 0.0, 0.0)
    _lib.check(lib.gd_guidance_divergence(_lib.ptr(div), C.byref(desc), 0, 0, h, w, st),
               "gd_guidance_divergence")
    compressed = torch.zeros_like(div)
    from .solvers import DCT_MAX_SIDE, _dct_plan
    if 2 <= min(h, w) and max(h, w) <= DCT_MAX_SIDE:
        # the reference's exact transform solve (solvers.py:224-262)
        (dct or _dct_plan(h, w)).solve(div, compressed)
    else:
        plan = cached_plan((Instance(h, w, "neumann", True),),
                           SolveParams(tolerance=NEUMANN_TOLERANCE, zero_start=True))
        plan.solve([div], [compressed], scale=-1.0)
    image = torch.empty_like(rad)
    out = torch.empty_like(rad)
    _lib.check(lib.gd_tm_compose(_lib.ptr(out), _lib.ptr(image), _lib.ptr(rad), _lib.ptr(lum),
                                 _lib.ptr(compressed), h, w, float(config.saturation), 99.5,
                                 _lib.ptr(scratch), st), "gd_tm_compose")
    return out, factor


def tone_map(radiance, config: ToneMapConfig | None = None):
    """Compress a linear HDR radiance map (h, w, 3) to display values in [0, 1].

    Returns the image and the attenuation factor that was applied.  Raises
    ``ValueError`` if the input is not a three-channel image.
    """
    config = config or ToneMapConfig()
    radiance = np.asarray(radiance, dtype=float)
    if radiance.ndim != 3 or radiance.shape[2] != 3:
        raise ValueError("tone mapping expects a three-channel radiance map")
    out, factor = tone_map_device(upload(radiance, _lib.device(), np.float64), config)
    return download(out), download(factor)
