"""The C ABI library loads without a GPU and exports every entry point that
include/tpsc_b200.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "tpsc_b200.h")
LIB = os.path.join(ROOT, "tpsc_conductivity_b200", "libtpsc_b200.so")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tpsc_[a-zA-Z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from tpsc_conductivity_b200 import build

        build.build()
    return ctypes.CDLL(LIB)


def test_header_declares_entry_points():
    names = declared()
    assert "tpsc_create" in names and "tpsc_solve" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_matches_header():
    from tpsc_conductivity_b200 import _lib

    assert sorted(n for n, _, _ in _lib.SIGNATURES) == declared()


def test_create_without_device_fails_cleanly(lib):
    """On a host with no CUDA device, tpsc_create returns NULL with a status."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib.tpsc_create.restype = ctypes.c_void_p
    st = ctypes.c_int(-1)
    h = lib.tpsc_create(0, ctypes.byref(st))
    assert not h and st.value != 0
