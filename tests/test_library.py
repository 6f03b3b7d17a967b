"""CPU checks of the C-ABI library: it loads and exports every declared symbol."""

from __future__ import annotations

import ctypes
import os
import re

import pytest

from gradient_domain_b200 import _lib, build

HEADER = os.path.join(os.path.dirname(build.HERE), "include", "gd_poisson.h")


def declared_functions() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gd_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(_lib.EXPORTS)


def test_library_builds_and_exports_every_symbol():
    path = build.build()
    lib = ctypes.CDLL(path)
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert b"sm_100a" in _lib.lib().gd_version()


def test_no_gpu_means_loud_failure(monkeypatch):
    import torch
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(_lib.GDError):
        _lib.device()


def test_smoother_argument_checks_run_on_the_host():
    """gd_rbgs_smooth rejects bad arguments before touching a device (dummy, never
    dereferenced pointers: every call below fails its checks first)."""
    fn = _lib.lib().gd_rbgs_smooth
    u, out, b = 256, 512, 768
    assert fn(None, out, b, 8, 8, 8, 0, 1.0, 1, None) == -1
    assert fn(u, u, b, 8, 8, 8, 0, 1.0, 1, None) == -1           # out is u
    assert fn(u, b, b, 8, 8, 8, 0, 1.0, 1, None) == -1           # out is b
    assert fn(u, out, b, 8, 8, 7, 0, 1.0, 1, None) == -1         # pitch below the width
    assert fn(u, out, b, 0, 8, 8, 0, 1.0, 1, None) == -1
    assert fn(u, out, b, 8, 8, 8, 3, 1.0, 1, None) == -1         # element type flag
    for sweeps in (0, 5, -1):
        assert fn(u, out, b, 8, 8, 8, 0, 1.0, sweeps, None) == -1
        assert b"sweeps" in _lib.lib().gd_last_error()


def test_plan_flags_are_checked_on_the_host():
    """gd_plan_create rejects launch-mode flags outside {0, 1} before it allocates
    anything or touches a device."""
    from gradient_domain_b200.plan import SolveParams
    grids = (_lib.GridDesc * 1)(_lib.GridDesc(64, 64, _lib.GD_NEUMANN, 1))
    out = ctypes.c_void_p()
    for field in ("dependent_launch", "persistent_coarse"):
        prm = SolveParams(zero_start=True).c_params()
        setattr(prm, field, 2)
        rc = _lib.lib().gd_plan_create(grids, 1, ctypes.byref(prm), ctypes.byref(out))
        assert rc == -1 and not out.value
        assert field.encode() in _lib.lib().gd_last_error()
