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


def test_sweep_points_are_the_seeded_workload():
    """tpsc_sweep_points (host only): deterministic for a seed, every point in
    the ranges of the sweep, Nw0 = 2 nextpow2(ceil(40 / (pi T)))."""
    import numpy as np

    from tpsc_conductivity_b200.api import sweep_points

    a = sweep_points(512)
    b = sweep_points(512)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, sweep_points(512, seed=1))
    nk0, nw0, n, T, tp, tpp, t3, U = a.T
    assert set(nk0.astype(int)) <= {32, 64, 128, 256} and len(set(nk0.astype(int))) == 4
    assert np.all((U >= 1) & (U <= 6)) and np.all((n >= 0.7) & (n <= 1.0))
    assert np.all((T >= 0.03) & (T <= 0.5)) and np.all((tp >= -0.3) & (tp <= 0))
    assert np.all(tpp == 0) and np.all(t3 == 0)
    pos = nw0 / 2
    need = np.ceil(40 / (np.pi * T))
    assert np.all(pos >= need) and np.all(pos / 2 < need)
    assert np.all(np.log2(nw0) == np.round(np.log2(nw0)))


def test_batch_create_without_device_fails_cleanly(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib.tpsc_batch_create.restype = ctypes.c_void_p
    st = ctypes.c_int(-1)
    assert not lib.tpsc_batch_create(0, 4, ctypes.byref(st)) and st.value != 0


def test_model_calls_reject_a_null_context(lib):
    """Entry points that need a model return TPSC_ERR_ARG (1) for a NULL
    context before any device call, with the reason in tpsc_last_error(NULL)
    (a null context or argument)."""
    import numpy as np

    from tpsc_conductivity_b200 import _lib

    lib.tpsc_last_error.restype = ctypes.c_char_p
    d = np.zeros(64)
    p = d.ctypes.data_as(ctypes.c_void_p)
    calls = {
        "tpsc_solve": (),
        "tpsc_sumrule_tangents": (p,),
        "tpsc_sumrule_vjp": (p, p),
        "tpsc_sigma_iqn": (ctypes.c_int(1), p, p),
        "tpsc_sigma_iqn_fd": (ctypes.c_int(1), p, p, p),
        "tpsc_chijj": (ctypes.c_int(1),),
    }
    for name, args in calls.items():
        assert getattr(lib, name)(None, *args) == _lib.ERR_ARG, name
        assert b"null" in lib.tpsc_last_error(None), name


def test_slice_plan_arguments_and_defaults(lib):
    """tpsc_set_slice_plan / tpsc_get_slice_plan are host-side settings: bad
    kinds, plans and lattices are rejected with TPSC_ERR_ARG, the folded
    matrix plan only where its tables exist (nk0 64, 128, 256), and the
    defaults are the FFT plan except the Sigma slice at nk0 = 256."""
    from tpsc_conductivity_b200 import _lib

    for kind, nk0, plan in [(4, 256, 1), (-1, 256, 0), (3, 256, 3), (3, 32, 1), (3, 100, 0), (0, 16, 1),
                            (0, 256, 2), (1, 256, 2), (3, 128, 2)]:
        assert lib.tpsc_set_slice_plan(kind, nk0, plan) == _lib.ERR_ARG, (kind, nk0, plan)
    assert lib.tpsc_get_slice_plan(4, 256) < 0
    assert lib.tpsc_get_slice_plan(3, 100) < 0
    assert lib.tpsc_get_slice_plan(3, 256) in (0, 1, 2)
    for kind in range(3):
        assert lib.tpsc_get_slice_plan(kind, 256) in (0, 1)
    for nk0 in (8, 16, 32):
        for kind in range(4):
            assert lib.tpsc_get_slice_plan(kind, nk0) == 0
    # a set plan reads back, and the default can be put back
    assert lib.tpsc_set_slice_plan(3, 128, 1) == 0
    assert lib.tpsc_get_slice_plan(3, 128) == 1
    assert lib.tpsc_set_slice_plan(3, 128, 0) == 0
    assert lib.tpsc_get_slice_plan(3, 128) == 0
