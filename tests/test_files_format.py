"""The reference's saved-run formats (chi0 binary, self_bin, self_tpsc ascii,
Green ascii): files written by the reference's own methods (the
files_l16_w32 fixture, tests/golden/make_golden.py) are read by this
library's readers, and its writers, given the same arrays, reproduce them
byte for byte under the reference's file names.  Host code only: no device."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import load_golden


@pytest.fixture(scope="module")
def lib():
    from tpsc_conductivity_b200 import _lib

    return _lib.load()


@pytest.fixture(scope="module")
def fx():
    g = load_golden("files_l16_w32")
    names = [str(n) for n in g["file_names"]]
    files = {n: bytes(g[f"file_{i}"]) for i, n in enumerate(names)}
    U, tp, tpp, t3, n, T, nk0, Nw0 = g["params"]
    sc = dict(zip([str(s) for s in g["scalars_names"]], g["scalars"]))
    return dict(g=g, files=files, U=U, tp=tp, tpp=tpp, t3=t3, n=n, T=T, nk0=int(nk0), Nw0=int(Nw0), sc=sc)


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _name(lib, fx, kind, l=0, m=0):
    buf = C.create_string_buffer(256)
    rc = lib.tpsc_file_name(kind, buf, 256, fx["U"], fx["tp"], fx["tpp"], fx["t3"], fx["n"], fx["T"], fx["nk0"],
                            fx["Nw0"], l, m)
    assert rc == 0
    name = buf.value.decode()
    assert name.startswith("./")
    return name[2:]


def _roundtrip(tmp_path, fx, name, write):
    path = str(tmp_path / name).encode()
    assert write(path) == 0
    with open(path, "rb") as f:
        assert f.read() == fx["files"][name]


def test_file_names_are_the_references(lib, fx):
    from tpsc_conductivity_b200 import _lib

    want = {_name(lib, fx, _lib.FILE_CHI0_BIN), _name(lib, fx, _lib.FILE_SELF_BIN),
            _name(lib, fx, _lib.FILE_SELF_ASCII), _name(lib, fx, _lib.FILE_GREEN, 2, 1)}
    assert want == set(fx["files"])
    buf = C.create_string_buffer(8)
    assert lib.tpsc_file_name(0, buf, 8, 1.0, 0, 0, 0, 0.9, 0.1, 8, 16, 0, 0) == _lib.ERR_ARG


def test_chi0_binary(lib, fx, tmp_path):
    from tpsc_conductivity_b200 import _lib

    name = _name(lib, fx, _lib.FILE_CHI0_BIN)
    src = tmp_path / ("in_" + name)
    src.write_bytes(fx["files"][name])
    nbq, nwmax = C.c_int(), C.c_int()
    assert lib.tpsc_read_chi0_bin(str(src).encode(), C.byref(nbq), C.byref(nwmax), None, 0) == 0
    nbk = fx["nk0"] // 2 + 1
    n8 = nbk * (nbk + 1) // 2
    assert (nbq.value, nwmax.value) == (nbk, fx["Nw0"] // 2)
    chi = np.zeros((nwmax.value + 1, n8))
    assert lib.tpsc_read_chi0_bin(str(src).encode(), C.byref(nbq), C.byref(nwmax), _dp(chi), chi.size - 1) == _lib.ERR_ARG
    assert lib.tpsc_read_chi0_bin(str(src).encode(), C.byref(nbq), C.byref(nwmax), _dp(chi), chi.size) == 0
    assert np.array_equal(chi, fx["g"]["chiqw"])
    _roundtrip(tmp_path, fx, name, lambda p: lib.tpsc_write_chi0_bin(p, nbq.value, nwmax.value, _dp(chi)))


def test_self_binary(lib, fx, tmp_path):
    from tpsc_conductivity_b200 import _lib

    name = _name(lib, fx, _lib.FILE_SELF_BIN)
    src = tmp_path / ("in_" + name)
    src.write_bytes(fx["files"][name])
    nbk, nbw = fx["nk0"] // 2 + 1, fx["Nw0"]
    n8 = nbk * (nbk + 1) // 2
    S = np.zeros((nbw // 2 + 1, n8), dtype=np.complex128)
    assert lib.tpsc_read_self_bin(str(src).encode(), nbk, nbw, _dp(S.view(np.float64))) == 0
    assert np.array_equal(S[:-1], fx["g"]["self"])
    # the last frame: (Sigma(k, beta/2), 0), left by the reference's Sigma stage
    assert not S[-1].imag.any() and S[-1].real.all()
    Sw, last = np.ascontiguousarray(S[:-1]), np.ascontiguousarray(S[-1])
    _roundtrip(tmp_path, fx, name, lambda p: lib.tpsc_write_self_bin(p, nbk, nbw, _dp(Sw.view(np.float64)),
                                                                     _dp(last.view(np.float64))))
    z = tmp_path / "zero_last.dat"
    assert lib.tpsc_write_self_bin(str(z).encode(), nbk, nbw, _dp(Sw.view(np.float64)), None) == 0
    assert z.read_bytes()[: Sw.nbytes] == fx["files"][name][: Sw.nbytes] and not any(z.read_bytes()[Sw.nbytes:])
    assert lib.tpsc_read_self_bin(b"/nonexistent/self_bin.dat", nbk, nbw, _dp(S.view(np.float64))) == _lib.ERR_ARG


def test_self_ascii(lib, fx, tmp_path):
    from tpsc_conductivity_b200 import _lib

    name = _name(lib, fx, _lib.FILE_SELF_ASCII)
    src = tmp_path / ("in_" + name)
    src.write_bytes(fx["files"][name])
    nbk, nbw = fx["nk0"] // 2 + 1, fx["Nw0"]
    n8 = nbk * (nbk + 1) // 2
    S = np.zeros((nbw // 2, n8), dtype=np.complex128)
    assert lib.tpsc_read_self_ascii(str(src).encode(), nbk, nbw, _dp(S.view(np.float64))) == 0
    # 17 significant digits: the values come back exactly
    assert np.array_equal(S, fx["g"]["self"])
    _roundtrip(tmp_path, fx, name, lambda p: lib.tpsc_write_self_ascii(p, nbk, nbw, 0, _dp(S.view(np.float64))))
    # a truncated file is an error, not a partial load
    short = tmp_path / "short.dat"
    short.write_bytes(fx["files"][name][: len(fx["files"][name]) // 2])
    assert lib.tpsc_read_self_ascii(str(short).encode(), nbk, nbw, _dp(S.view(np.float64))) == _lib.ERR_ARG


def test_green_ascii(lib, fx, tmp_path):
    from tpsc_conductivity_b200 import _lib

    name = _name(lib, fx, _lib.FILE_GREEN, 2, 1)
    g = fx["g"]
    nbk = fx["nk0"] // 2 + 1
    l, m = 2, 1
    o = m + l * (l + 1) // 2
    # hamiltonien::ek_val(2, 1) - mu (src/hamiltonien.cpp:107-116), the mu of find_mu
    ek_mu = g["ek"][2, 1] - fx["sc"]["mu"]
    S = np.ascontiguousarray(g["self"])
    col = S[:, o:]
    _roundtrip(tmp_path, fx, name, lambda p: lib.tpsc_write_green_ascii(
        p, fx["Nw0"], fx["T"], ek_mu, fx["sc"]["Sigma_inf"], g["sigma_inf2"][o], g["sigma_inf3"][o],
        _dp(col.view(np.float64)), S.shape[1]))
