"""GPU parity of the temporally blocked red-black Gauss-Seidel smoother (gd_rbgs_smooth).

The kernel evaluates multigrid._smooth's expression (multigrid.py:147-165) in
the same order with round-to-nearest operations, so every comparison here is
bitwise: FP64 against the reference's own output (golden vectors) and the
oracle, FP32 against the same expression evaluated in float32.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch
import torch.nn.functional as F

import gradient_domain_b200 as gd
from gradient_domain_b200 import _lib
from oracle import multigrid as om

pytestmark = pytest.mark.gpu

SMOOTH_CASES = ["sm37x53", "sm37x53s3", "sm5x131", "sm70x260s6"]


@pytest.mark.parametrize("name", SMOOTH_CASES)
def test_smooth_matches_reference_golden_bitwise(golden, name):
    sweeps, h = golden[f"{name}_opts"]
    u0, b = golden[f"{name}_u0"], golden[f"{name}_b"]
    got64 = gd.smooth(u0, b, float(h), int(sweeps))
    got32 = gd.smooth(u0.astype(np.float32), b.astype(np.float32), float(h), int(sweeps))
    assert got64.dtype == np.float64 and got32.dtype == np.float32
    np.testing.assert_array_equal(got64, golden[f"{name}_f64"])
    np.testing.assert_array_equal(got32, golden[f"{name}_f32"])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("shape", [(1, 1), (2, 3), (3, 1), (1, 200), (129, 131), (300, 509),
                                   (64, 1000), (517, 243)])
def test_smooth_matches_oracle_bitwise(shape, dtype):
    rng = np.random.default_rng(shape[0] * 1000 + shape[1])
    u0 = rng.standard_normal(shape).astype(dtype)
    b = rng.standard_normal(shape).astype(dtype)
    for sweeps in (1, 2, 3, 4, 5):
        got = gd.smooth(u0, b, 0.6, sweeps)
        ref = om.smooth(u0, b, 0.6, sweeps)
        assert got.dtype == ref.dtype == dtype
        np.testing.assert_array_equal(got, ref, err_msg=f"{shape} sweeps={sweeps}")
    np.testing.assert_array_equal(gd.smooth(u0, b, 0.6, 0), u0)


def _torch_smooth(u, b, h2, sweeps):
    """The reference expression on the device, one elementwise op at a time."""
    ny, nx = u.shape
    ii = torch.arange(ny, device=u.device)[:, None]
    jj = torch.arange(nx, device=u.device)[None, :]
    colour = (ii + jj) % 2
    for _ in range(sweeps):
        for parity in (0, 1):
            p = F.pad(u[None, None], (1, 1, 1, 1))[0, 0]
            nb = p[:-2, 1:-1] + p[2:, 1:-1]
            nb = nb + p[1:-1, :-2]
            nb = nb + p[1:-1, 2:]
            cand = 0.25 * (nb - h2 * b)
            u = torch.where(colour == parity, cand, u)
    return u


@pytest.mark.parametrize("n,sweeps", [(4096, 1), (2048, 4)])
def test_smooth_full_size_fp32_bitwise(n, sweeps):
    dev = _lib.device()
    g = torch.Generator(device=dev).manual_seed(n + sweeps)
    u = torch.randn((n, n), device=dev, generator=g)
    b = torch.randn((n, n), device=dev, generator=g)
    got = gd.smooth(u, b, 1.0, sweeps)
    assert got.device.type == "cuda" and got.dtype == torch.float32
    ref = _torch_smooth(u, b, 1.0, sweeps)
    assert torch.equal(got, ref)


@pytest.mark.parametrize("fp64", [0, 1])
@pytest.mark.parametrize("pitch_pad,offset", [(0, 0), (3, 0), (4, 1), (8, 0)])
def test_smooth_any_pitch_and_alignment(fp64, pitch_pad, offset):
    """Rows at any pitch and start (vector and scalar paths); padding is never written."""
    dev = _lib.device()
    ny, nx = 75, 261
    pitch = nx + pitch_pad
    dtype = torch.float64 if fp64 else torch.float32
    npdt = np.float64 if fp64 else np.float32
    rng = np.random.default_rng(pitch * 10 + offset)
    u0 = rng.standard_normal((ny, nx)).astype(npdt)
    b = rng.standard_normal((ny, nx)).astype(npdt)

    def pitched(a, fill):
        buf = torch.full((offset + ny * pitch,), fill, dtype=dtype, device=dev)
        view = buf[offset:].view(ny, pitch)
        if a is not None:
            view[:, :nx] = torch.as_tensor(a, device=dev)
        return buf, view

    ub, uv = pitched(u0, 0.0)
    bb, bv = pitched(b, 0.0)
    ob, ov = pitched(None, 7.0)
    for sweeps in (1, 2, 3, 4):
        ov.fill_(7.0)
        rc = _lib.lib().gd_rbgs_smooth(_lib.ptr(uv), _lib.ptr(ov), _lib.ptr(bv), ny, nx, pitch,
                                       fp64, 1.5, sweeps, _lib.stream_handle())
        _lib.check(rc, "gd_rbgs_smooth")
        torch.cuda.synchronize()
        got = ov[:, :nx].cpu().numpy()
        np.testing.assert_array_equal(got, om.smooth(u0, b, 1.5, sweeps))
        if pitch_pad:
            assert bool((ov[:, nx:] == 7.0).all()), "padding columns were written"


def test_smooth_rejects_bad_arguments():
    dev = _lib.device()
    u = torch.zeros((16, 16), device=dev)
    out = torch.zeros_like(u)
    fn = _lib.lib().gd_rbgs_smooth
    s = _lib.stream_handle()
    p = _lib.ptr
    assert fn(p(u), p(u), p(u), 16, 16, 16, 0, 1.0, 1, s) == -1      # out is u
    assert fn(p(u), p(out), p(out), 16, 16, 16, 0, 1.0, 1, s) == -1  # out is b
    assert fn(p(u), p(out), p(u), 16, 16, 16, 0, 1.0, 5, s) == -1    # too many sweeps per call
    assert b"sweeps" in _lib.lib().gd_last_error()
    assert fn(p(u), p(out), p(u), 16, 16, 16, 0, 1.0, 0, s) == -1
    assert fn(p(u), p(out), p(u), 0, 16, 16, 0, 1.0, 1, s) == -1
    assert fn(p(u), p(out), p(u), 16, 16, 15, 0, 1.0, 1, s) == -1    # pitch < width
    assert fn(p(u), p(out), p(u), 16, 16, 16, 2, 1.0, 1, s) == -1
    with pytest.raises(ValueError):
        gd.smooth(np.zeros((3, 4)), np.zeros((4, 3)))
