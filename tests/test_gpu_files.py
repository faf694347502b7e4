"""Saved-run files and warm starts on the GPU: the drop-in classes write the
reference's chi0 binary, self_bin, self_tpsc and Green files with the
reference's numbers (files_l16_w32 fixture, written by the reference's own
methods), read the reference's self_bin back into the device, and the C ABI's
setters (tpsc_set_self, tpsc_set_chi0) reproduce the reference's mu and chi0max
from the reference's own arrays."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "tpsc_conductivity_b200", "dropin", "_build", "files_main_b200")


def _fx():
    g = load_golden("files_l16_w32")
    names = [str(n) for n in g["file_names"]]
    return g, {n: bytes(g[f"file_{i}"]) for i, n in enumerate(names)}


def _args(g):
    U, tp, tpp, t3, n, T, nk0, Nw0 = g["params"]
    return [repr(float(x)) for x in (U, tp, tpp, t3, n, T)] + [str(int(nk0)), str(int(Nw0))]


def _run(mode, g, cwd):
    r = subprocess.run([BIN, mode] + _args(g), cwd=cwd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return [float(m) for m in re.findall(r"^mu (\S+)$", r.stdout, re.M)]


def _cplx(b, off=0):
    a = np.frombuffer(b, dtype=np.float64, offset=off)
    return a[0::2] + 1j * a[1::2]


@pytest.mark.skipif(not os.path.exists(BIN), reason="files_main_b200 is built by make -C tpsc_conductivity_b200/dropin")
def test_dropin_writes_the_reference_files(tmp_path):
    g, ref = _fx()
    mus = _run("save", g, tmp_path)
    sc = dict(zip([str(s) for s in g["scalars_names"]], g["scalars"]))
    assert len(mus) == 2 and abs(mus[0] - sc["mu"]) < 1e-9
    # the warm start from this program's own self_bin finds the same mu
    assert mus[1] == mus[0]
    got = {f: (tmp_path / f).read_bytes() for f in os.listdir(tmp_path)
           if f.startswith(("chi0_", "self_bin_", "self_tpsc_", "Green_"))
           and not f.startswith(("chi0_qmax_wn_", "chi0_wn0_q_"))}
    assert set(got) == set(ref)
    for name, want in ref.items():
        have = got[name]
        if name.startswith("chi0_"):
            assert len(have) == len(want) and have[:8] == want[:8]  # int nbq, int nwmax
            a, b = np.frombuffer(have, np.float64, offset=8), np.frombuffer(want, np.float64, offset=8)
            assert np.allclose(a, b, rtol=1e-9, atol=1e-12 * np.abs(b).max())
        elif name.startswith("self_bin_"):
            assert len(have) == len(want)
            a, b = _cplx(have), _cplx(want)
            assert np.allclose(a, b, rtol=1e-9, atol=1e-10 * np.abs(b).max())
        else:
            la, lb = have.decode().splitlines(), want.decode().splitlines()
            assert len(la) == len(lb)
            # the same fields starting at the same columns (setw(10) indices,
            # setw(25) real parts); values to 1e-9
            for x, y in zip(la, lb):
                assert [m.start() for m in re.finditer(r"\S+", x)] == [m.start() for m in re.finditer(r"\S+", y)]
            ta, tb = np.loadtxt(la, ndmin=2), np.loadtxt(lb, ndmin=2)
            ni = 3 if name.startswith("self_tpsc_") else 1
            assert np.array_equal(ta[:, :ni], tb[:, :ni])
            assert np.allclose(ta[:, ni:], tb[:, ni:], rtol=1e-9, atol=1e-10 * np.abs(tb[:, ni:]).max())


@pytest.mark.skipif(not os.path.exists(BIN), reason="files_main_b200 is built by make -C tpsc_conductivity_b200/dropin")
def test_dropin_reads_the_references_self_bin(tmp_path):
    g, ref = _fx()
    name = next(n for n in ref if n.startswith("self_bin_"))
    (tmp_path / name).write_bytes(ref[name])
    mus = _run("load", g, tmp_path)
    sc = dict(zip([str(s) for s in g["scalars_names"]], g["scalars"]))
    assert len(mus) == 1 and abs(mus[0] - sc["mu"]) < 1e-9


def test_abi_warm_start_from_the_references_arrays():
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Green

    g, ref = _fx()
    U, tp, tpp, t3, n, T, nk0, Nw0 = g["params"]
    sc = dict(zip([str(s) for s in g["scalars_names"]], g["scalars"]))
    gr = Green(int(nk0), int(Nw0), n, T, 0.1, (tp, tpp, t3, U))
    gr.solve()
    lib, h = gr.ctx.lib, gr.ctx.h
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    # Sigma(k, beta/2): the last frame of the reference's self_bin
    n8 = gr.dims()[3]
    mid = np.zeros(n8)
    assert lib.tpsc_get_sigma_tau(h, int(Nw0) // 2, dp(mid)) == 0
    name = next(n for n in ref if n.startswith("self_bin_"))
    last = _cplx(ref[name], 16 * n8 * (int(Nw0) // 2))
    assert np.allclose(mid, last.real, rtol=1e-9, atol=1e-10 * np.abs(last).max())
    # the reference's Sigma with its tails -> the reference's mu
    S = np.ascontiguousarray(g["self"])
    s2, s3, s4 = (np.ascontiguousarray(g[k]) for k in ("sigma_inf2", "sigma_inf3", "sigma_inf4"))
    sinf = np.array([sc["Sigma_inf"]])
    assert lib.tpsc_set_self(h, dp(S.view(np.float64)), dp(s2), dp(s3), dp(s4), dp(sinf)) == 0
    gr.find_mu()
    assert abs(gr.scalars()["mu"] - sc["mu"]) < 1e-10
    out = gr.self_energy()
    assert np.array_equal(out["S"], S) and np.array_equal(out["Sigma_inf2"], s2)
    # the reference's chi0 -> its chi0max and qmax
    chi = np.ascontiguousarray(g["chiqw"])
    assert lib.tpsc_set_chi0(h, dp(chi)) == 0
    s = gr.scalars()
    assert s["chi0max"] == sc["chi0max"] and (s["qmax0"], s["qmax1"]) == (sc["qmax0"], sc["qmax1"])
    assert np.array_equal(gr.chi0()["chiqw"], chi)
    # a NULL Sigma is refused
    assert lib.tpsc_set_self(h, None, None, None, None, None) == _lib.ERR_ARG


@pytest.mark.skipif(not os.path.exists(BIN), reason="files_main_b200 is built by make -C tpsc_conductivity_b200/dropin")
def test_dropin_corr_length_scan_writes_the_reference_file(tmp_path):
    """chi::calc_corr_length over n in {0.85, 0.9}, T in {0.2, 0.3}: the same
    corrLgth file as the reference's (corr_l16_w64 fixture) -- vF from the
    constructor's Fermi surface on every line, errUs = errUc = 0 as the
    reference leaves them, the integer columns exact, the rest to 1e-8."""
    g = load_golden("corr_l16_w64")
    name = str(g["file_names"][0])
    want = bytes(g["file_0"]).decode().splitlines()
    U, tp, tpp, t3, n, T, nk0, Nw0 = g["params"]
    args = [repr(float(x)) for x in (U, tp, tpp, t3, n, T)] + [str(int(nk0)), str(int(Nw0))]
    r = subprocess.run([BIN, "corr"] + args, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    have = (tmp_path / name).read_text().splitlines()
    assert len(have) == len(want) == 4
    for x, y in zip(have, want):
        assert [m.start() for m in re.finditer(r"\S+", x)] == [m.start() for m in re.finditer(r"\S+", y)]
    a, b = np.loadtxt(have, ndmin=2), np.loadtxt(want, ndmin=2)
    ints = [15, 16, 17]
    assert np.array_equal(a[:, ints], b[:, ints])
    assert not a[:, [5, 7]].any()
    assert len(set(a[:, 3])) == 1
    fl = [c for c in range(a.shape[1]) if c not in ints]
    assert np.allclose(a[:, fl], b[:, fl], rtol=1e-8, atol=1e-12)


@pytest.mark.skipif(not os.path.exists(BIN), reason="files_main_b200 is built by make -C tpsc_conductivity_b200/dropin")
def test_dropin_self_re_w_bz_writes_the_reference_files(tmp_path):
    """green::calc_Self_Re_w_BZ: for every k of the reduced zone, the Pade and
    J-fraction Sigma(k, w + i eta) and A(k, w) files of the reference
    (rew_l16_w64, 76 files), with the same names and columns.
    * The J-fraction continues from 4 points and is well conditioned: its
      files agree to 1e-8 of each file's scale (measured 2e-10).
    * The plain Pade runs a 16-point continued fraction out to w = +-4.  Two
      FP64 evaluations of that same recursion on the SAME Sigma differ by up
      to ~1e-4 of the scale: the device recursion on the reference's own
      Sigma gives median 1.5e-6, max 1.1e-4.  Those files are therefore held
      to a median of 1e-5 and a maximum of 1e-3."""
    g = load_golden("rew_l16_w64")
    names = [str(n) for n in g["file_names"]]
    U, tp, tpp, t3, n, T, nk0, Nw0 = g["params"]
    args = [repr(float(x)) for x in (U, tp, tpp, t3, n, T)] + [str(int(nk0)), str(int(Nw0))]
    r = subprocess.run([BIN, "rew"] + args, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    got = sorted(f for f in os.listdir(tmp_path) if f.startswith(("Self_Re_w_", "spectr_wgt_")))
    assert got == sorted(names)
    pade = []
    for i, name in enumerate(names):
        want = bytes(g[f"file_{i}"]).decode().splitlines()
        have = (tmp_path / name).read_text().splitlines()
        assert len(have) == len(want) == 9
        for x, y in zip(have, want):
            assert [m.start() for m in re.finditer(r"\S+", x)][:2] == [m.start() for m in re.finditer(r"\S+", y)][:2]
        a, b = np.loadtxt(have, ndmin=2), np.loadtxt(want, ndmin=2)
        assert a.shape == b.shape and np.array_equal(a[:, 0], b[:, 0])
        err = np.abs(a[:, 1:] - b[:, 1:]).max() / np.abs(b[:, 1:]).max()
        if "Jfrac" in name:
            assert err < 1e-8, (name, err)
        else:
            pade.append(err)
    assert len(pade) == 38 and np.median(pade) < 1e-5 and max(pade) < 1e-3


@pytest.mark.skipif(not os.path.exists(BIN), reason="files_main_b200 is built by make -C tpsc_conductivity_b200/dropin")
def test_dropin_edc_writes_the_reference_files(tmp_path):
    """green::EDC, both overloads (edc_l16_w32, written by the reference on
    one OpenMP thread): the non-uniform-grid Pade over the reduced zone and
    over a k list (folded into the zone, as the file names show) to 1e-8 of
    each file's scale, and the 16-point Pade on w = -10..10 to 1e-7; the same
    file names."""
    g = load_golden("edc_l16_w32")
    names = [str(n) for n in g["file_names"]]
    U, tp, tpp, t3, n, T, nk0, Nw0 = g["params"]
    args = [repr(float(x)) for x in (U, tp, tpp, t3, n, T)] + [str(int(nk0)), str(int(Nw0))]
    r = subprocess.run([BIN, "edc"] + args, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert sorted(f for f in os.listdir(tmp_path) if f.startswith("edc")) == sorted(names)
    assert any(nm.startswith("edcl_") and nm.endswith("_3_1_-2.0e+00_2.0e+00.dat") for nm in names)
    for i, name in enumerate(names):
        b = np.loadtxt(bytes(g[f"file_{i}"]).decode().splitlines(), ndmin=2)
        a = np.loadtxt((tmp_path / name).read_text().splitlines(), ndmin=2)
        assert a.shape == b.shape and np.array_equal(a[:, 0], b[:, 0])
        err = np.abs(a[:, 1:] - b[:, 1:]).max() / np.abs(b[:, 1:]).max()
        assert err < (1e-7 if name.startswith("edc2") else 1e-8), (name, err)


@pytest.mark.skipif(not os.path.exists(BIN), reason="files_main_b200 is built by make -C tpsc_conductivity_b200/dropin")
def test_dropin_infinite_lattice_chi0(tmp_path):
    """chi0::calc_chi0_qlims (the infinite lattice, which the reference
    integrates adaptively to ~1e-10) from lattice sums doubled until they
    converge: the same chi0_q files (q columns exact, chi0 to 1e-9), the same
    infinite-system mu0 (1e-9), and chiqw_discret on the 16x16 lattice
    (1e-12)."""
    g = load_golden("chi0inf_l16")
    names = [str(n) for n in g["file_names"]]
    U, tp, tpp, t3, n, T, nk0, Nw0 = g["params"]
    args = [repr(float(x)) for x in (U, tp, tpp, t3, n, T)] + [str(int(nk0)), str(int(Nw0))]
    r = subprocess.run([BIN, "chi0inf"] + args, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    val = {k: float(v) for k, v in re.findall(r"^(chi_discret|mu0_finite|mu0_inf) (\S+)$", r.stdout, re.M)}
    assert abs(val["chi_discret"] - float(g["chi_discret"])) < 1e-12 * abs(float(g["chi_discret"]))
    assert abs(val["mu0_finite"] - float(g["mu0_finite"])) < 1e-10
    assert abs(val["mu0_inf"] - float(g["mu0_inf"])) < 1e-9
    assert sorted(f for f in os.listdir(tmp_path) if f.startswith("chi0_q_")) == sorted(names)
    for i, name in enumerate(names):
        want = bytes(g[f"file_{i}"]).decode().splitlines()
        have = (tmp_path / name).read_text().splitlines()
        assert len(have) == len(want) == 6
        for x, y in zip(have, want):
            assert x.split()[:2] == y.split()[:2]
        a, b = np.loadtxt(have, ndmin=2), np.loadtxt(want, ndmin=2)
        assert np.allclose(a[:, 2], b[:, 2], rtol=1e-9, atol=1e-12), (name, a[:, 2] - b[:, 2])
