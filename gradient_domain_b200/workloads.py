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
* ``batch_instances``: the uneven batch of integration and compositing
  problems (sides 64-2048, one or three channels).
"""

from __future__ import annotations

import numpy as np



def _downsample(image):
    """5-tap binomial blur with edge replication, every other sample."""
    k = np.array([1.0, 4.0, 6.0, 4.0, 1.0]) / 16.0
    p = np.pad(image, ((0, 0), (2, 2)), mode="edge")
    b = sum(kk * p[:, i:i + image.shape[1]] for i, kk in enumerate(k))
    p = np.pad(b, ((2, 2), (0, 0)), mode="edge")
    b = sum(kk * p[i:i + image.shape[0], :] for i, kk in enumerate(k))
    return b[::2, ::2]


def _attenuation(log_r, alpha=0.1, beta=0.85, levels=1, eps=1e-4):
    """Host copy of the attenuation factor used to shape the synthetic field
    (one pyramid level by default, as the tone-mapping workload uses)."""
    pyr = [log_r]
    while len(pyr) < levels and min(pyr[-1].shape) > 16:
        pyr.append(_downsample(pyr[-1]))
    if len(pyr) != 1:
        raise NotImplementedError("the synthetic workload uses a single level")
    p = np.pad(log_r, 1, mode="edge")
    gx = (p[1:-1, 2:] - p[1:-1, :-2]) / 2.0
    gy = (p[2:, 1:-1] - p[:-2, 1:-1]) / 2.0
    m = np.sqrt(gx * gx + gy * gy)
    scale = alpha * max(float(m.mean()), eps)
    fl = np.maximum(m, eps)
    return (scale / fl) * (fl / scale) ** beta


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
    for c in range(channels):
        mod = 0.05 + blob_image((size, size), 64, rng, sigma=(10.0 * scale, 120.0 * scale),
                                noise=0.0)
        log_r = 2.5 * rng.standard_normal((size, size)) + np.log(mod)
        factor = _attenuation(log_r)
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


def masked_system(source, target, mask, crop=True):
    """Masked Poisson system of seamless cloning in "import" mode at offset (0, 0).

    Returns (f, unknown, window): per-channel right-hand sides of the reference
    sign convention A x = f (A positive), the unknown mask and the window they
    cover.  With ``crop`` the window is the bounding box of the unknowns plus a
    one-pixel ring, otherwise the whole canvas.  The system is the one
    poisson.py:154-244 assembles for
    seamless_clone(source, target, mask, (0, 0), mode="import", domain="mask").
    """
    inner = np.zeros(mask.shape, dtype=bool)
    inner[1:-1, 1:-1] = mask[1:-1, 1:-1]
    if crop:
        rows = np.nonzero(inner.any(axis=1))[0]
        cols = np.nonzero(inner.any(axis=0))[0]
        win = (slice(rows[0] - 1, rows[-1] + 2), slice(cols[0] - 1, cols[-1] + 2))
    else:
        win = (slice(0, mask.shape[0]), slice(0, mask.shape[1]))
    unk = inner[win]
    f = []
    for c in range(target.shape[2]):
        sgx, sgy = forward_gradient(source[..., c])
        tgx, tgy = forward_gradient(target[..., c])
        gx = np.where(mask, sgx, tgx)[win]
        gy = np.where(mask, sgy, tgy)[win]
        div = divergence(gx, gy)
        img = target[..., c][win]
        b = div.copy()
        # subtract known neighbour values (the order of poisson.py:218-224)
        for dy, dx in ((-1, 0), (1, 0), (0, -1), (0, 1)):
            nb_unk = np.roll(np.roll(unk, -dy, axis=0), -dx, axis=1)
            nb_val = np.roll(np.roll(img, -dy, axis=0), -dx, axis=1)
            b = np.where(unk & ~nb_unk, b - nb_val, b)
        f.append(np.where(unk, -b, 0.0))
    return np.stack(f), unk, win


def blob_pair(shape, channels, rng):
    """Source and target images (h, w, channels) in [0, 1], sums of 32 blobs each."""
    m = min(shape)

    def image():
        img = np.stack([blob_image(shape, 32, rng, sigma=(0.005 * m + 1.0, 0.06 * m + 1.0))
                        for _ in range(channels)], axis=2)
        img -= img.min()
        return img / max(img.max(), 1e-12)

    return image(), image()


def batch_instances(count=256, seed=3, side=(64, 2048)):
    """The uneven batch: `count` images of 1 or 3 channels (p = 0.5).

    Sides are log-uniform in [64, 2048], the aspect ratio uniform in [0.5, 2],
    both sides rounded to multiples of 8.  Even-numbered images are Neumann
    integrations of a blob gradient field (the single-image integration case),
    odd ones seamless composites: a blob source pasted into a blob target
    inside a 12-vertex star polygon (radii 0.15-0.45 of the shorter side), the
    masked system of the compositing case on the whole canvas.  Returns a list
    of dicts with keys boundary, f (c, h, w) and, for masks, unknown (h, w),
    source and target (h, w, c).
    """
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        s = float(np.exp(rng.uniform(np.log(side[0]), np.log(side[1]))))
        aspect = rng.uniform(0.5, 2.0)
        h = max(8, int(round(s * np.sqrt(aspect) / 8.0)) * 8)
        w = max(8, int(round(s / np.sqrt(aspect) / 8.0)) * 8)
        ch = 1 if rng.random() < 0.5 else 3
        if k % 2 == 0:
            f = np.stack([-neumann_blobs_shape((h, w), rng) for _ in range(ch)])
            out.append({"boundary": "neumann", "f": f})
        else:
            m = min(h, w)
            mask = star_polygon_mask_shape((h, w), rng, rmin=0.15 * m, rmax=0.45 * m)
            source, target = blob_pair((h, w), ch, rng)
            f, unk, _ = masked_system(source, target, mask, crop=False)
            out.append({"boundary": "masked", "f": f, "unknown": unk, "source": source,
                        "target": target})
    return out


def neumann_blobs_shape(shape, rng):
    src = blob_image(shape, 32, rng, sigma=(0.01 * min(shape), 0.12 * min(shape)))
    return divergence(*forward_gradient(src))


def star_polygon_mask_shape(shape, rng, vertices=12, rmin=10.0, rmax=40.0):
    """Star polygon centred in an (h, w) canvas, rasterised at pixel centres."""
    h, w = shape
    ang = 2 * np.pi * np.arange(vertices) / vertices + rng.uniform(-0.2, 0.2, vertices)
    rad = rng.uniform(rmin, rmax, vertices)
    vy, vx = h / 2.0 + rad * np.sin(ang), w / 2.0 + rad * np.cos(ang)
    yy = np.arange(h)[:, None] + 0.5
    xx = np.arange(w)[None, :] + 0.5
    inside = np.zeros((h, w), dtype=bool)
    j = vertices - 1
    for i in range(vertices):
        crosses = (vy[i] > yy) != (vy[j] > yy)
        with np.errstate(divide="ignore", invalid="ignore"):
            xint = (vx[j] - vx[i]) * (yy - vy[i]) / (vy[j] - vy[i]) + vx[i]
        inside ^= crosses & (xx < xint)
        j = i
    return inside
