"""tpsc_fma_peak: the FMA throughput the transform kernels' roofline is set
against -- positive, FP32 above FP64, and within the B200's nominal range."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def test_fma_peaks():
    from tpsc_conductivity_b200 import _lib

    lib = _lib.load()
    v64, v32 = C.c_double(), C.c_double()
    assert lib.tpsc_fma_peak(64, C.byref(v64)) == 0
    assert lib.tpsc_fma_peak(32, C.byref(v32)) == 0
    assert 1.0 < v64.value < 200.0 and 10.0 < v32.value < 400.0
    assert v32.value > v64.value
    assert lib.tpsc_fma_peak(16, C.byref(v64)) == _lib.ERR_ARG
