"""The C-ABI library loads and exports every symbol include/cloverb200.h declares.

No compute call is made here (no GPU is needed): only symbol lookup, the
argument checks that fail before touching a device, and the error path of
cb_create on a machine without a CUDA device.
"""
import ctypes
import os
import re

import pytest

import cloverleaf_b200 as cb
from cloverleaf_b200 import chunk as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "cloverb200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = cb.library()
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(C.EXPORTS) == names


def test_version_and_error_string():
    lib = cb.library()
    assert lib.cb_version() >= 1
    assert isinstance(lib.cb_last_error(), bytes)


def test_argument_checks_before_device():
    lib = cb.library()
    h = ctypes.c_void_p()
    assert lib.cb_create(0, 10, 0, 0, ctypes.byref(h)) == 1
    assert b"at least one cell" in lib.cb_last_error()
    assert lib.cb_create(10, 10, 7, 0, ctypes.byref(h)) == 1
    assert lib.cb_destroy(None) == 0
    assert lib.cb_ideal_gas(None, 0, 0) == 1


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(cb.CloverError):
        cb.Chunk(16, 16)
