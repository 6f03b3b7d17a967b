"""The allocation-free V-cycle entry point, checked against the allocating one.

``gd_ref_vcycle_static`` serves callers that cannot allocate device memory at
the moment they need a cycle (code inside CUDA stream capture, real-time loops
without allocation after start-up, plug-ins of applications that own the
memory budget).  Its scratch is a 4 MiB static device array shared by every
call.  This file is collected last so that a failure here comes after every
other test has run; it passes alone in a fresh process as well.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gradient_domain_b200 import _lib

pytestmark = pytest.mark.gpu

SHAPE = (127, 93)
OPTS = dict(pre=2, post=2, coarsest_size=8, coarsest_sweeps=60)


def _allocating(u, b, spacing):
    m, n = b.shape
    nbytes = int(_lib.lib().gd_ref_workspace_bytes(m, n, OPTS["coarsest_size"]))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=b.device)
    _lib.check(_lib.lib().gd_ref_vcycle(_lib.ptr(u), _lib.ptr(b), m, n, spacing, OPTS["pre"],
                                        OPTS["post"], OPTS["coarsest_size"],
                                        OPTS["coarsest_sweeps"], _lib.ptr(ws), nbytes,
                                        _lib.stream_handle()), "gd_ref_vcycle")


def _static(u, b, spacing):
    m, n = b.shape
    _lib.check(_lib.lib().gd_ref_vcycle_static(_lib.ptr(u), _lib.ptr(b), m, n, spacing,
                                               OPTS["pre"], OPTS["post"],
                                               OPTS["coarsest_size"], OPTS["coarsest_sweeps"],
                                               _lib.stream_handle()), "gd_ref_vcycle_static")


def test_static_vcycle_matches_allocating_vcycle_twice():
    dev = _lib.device()
    for call, spacing in enumerate((1.0, 0.5)):
        rng = np.random.default_rng(100 + call)
        b = torch.as_tensor(rng.standard_normal(SHAPE)).to(dev)
        u0 = torch.as_tensor(0.1 * rng.standard_normal(SHAPE)).to(dev)
        expected, got = u0.clone(), u0.clone()
        _allocating(expected, b, spacing)
        _static(got, b, spacing)
        torch.cuda.synchronize()
        # the same kernels in the same order: bitwise equal
        assert torch.equal(got, expected), call


def test_single_level_grids_need_no_scratch():
    """A grid that is already the coarsest (here its short side is coarsest_size) is
    smoothed in place without scratch, so it is accepted even when the allocating
    cycle's workspace for it would exceed the static array, and matches that cycle."""
    dev = _lib.device()
    m, n, sweeps = 70000, 8, 4
    assert _lib.lib().gd_ref_workspace_bytes(m, n, 8) > (4 << 20)
    rng = np.random.default_rng(7)
    b = torch.as_tensor(rng.standard_normal((m, n))).to(dev)
    expected, got = torch.zeros_like(b), torch.zeros_like(b)
    nbytes = int(_lib.lib().gd_ref_workspace_bytes(m, n, 8))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    _lib.check(_lib.lib().gd_ref_vcycle(_lib.ptr(expected), _lib.ptr(b), m, n, 1.0, 2, 2, 8,
                                        sweeps, _lib.ptr(ws), nbytes, _lib.stream_handle()),
               "gd_ref_vcycle")
    _lib.check(_lib.lib().gd_ref_vcycle_static(_lib.ptr(got), _lib.ptr(b), m, n, 1.0, 2, 2, 8,
                                               sweeps, _lib.stream_handle()),
               "gd_ref_vcycle_static")
    torch.cuda.synchronize()
    assert torch.equal(got, expected)


def test_static_vcycle_rejects_grids_beyond_its_scratch():
    dev = _lib.device()
    b = torch.zeros((1024, 1024), dtype=torch.float64, device=dev)
    u = torch.zeros_like(b)
    rc = _lib.lib().gd_ref_vcycle_static(_lib.ptr(u), _lib.ptr(b), 1024, 1024, 1.0, 2, 2, 8, 60,
                                         _lib.stream_handle())
    assert rc == -1
    assert b"static array" in _lib.lib().gd_last_error()
