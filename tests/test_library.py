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
