"""The current-current correlator on the GPU against the reference's own arrays.

cond_opt::calc_chijj_vertex_corr_all_optim (src/cond_opt.cpp:2537-4286), the
bubble + Maki-Thompson branch, run through the C ABI (tpsc_chijj) after a
full solve, compared with what the unmodified reference computed on the same
inputs (tests/golden/*.npz): chijj1 (bubble), chijj2 (vertex correction),
kx0 and, where the fixture has them, the angle-resolved sums.

Tolerance: 1e-10 of the largest |chi_jj| for the arrays, 1e-10 relative for
kx0.  The GPU sums in another order than the reference's OpenMP loops and its
splines are solved by a different (banded LU vs. Thomas) method; the oracle
restatement agrees with the reference to 1e-12 on the same cases.
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu

COND = [n for n in golden_names() if "chijj1" in load_golden(n)]
TOL = 1e-10


def _ntheta(g):
    return g["chijj1_k"].shape[1] if "chijj1_k" in g else 1


def _cond(p):
    from tpsc_conductivity_b200.api import CondOpt

    return CondOpt(p["nk0"], p["Nw0"], p["n"], p["T"], 0.1, (p["tp"], p["tpp"], p["t3"], p["U"]))


def _check(r, g):
    s1 = np.max(np.abs(g["chijj1"]))
    s2 = np.max(np.abs(g["chijj2"]))
    e1 = np.max(np.abs(r["chijj1"] - g["chijj1"])) / s1
    e2 = np.max(np.abs(r["chijj2"] - g["chijj2"])) / s2
    ek = abs(r["kx0"] - float(g["kx0"])) / abs(float(g["kx0"]))
    assert e1 <= TOL, e1
    assert e2 <= TOL, e2
    assert ek <= TOL, ek
    if "chijj1_k" in g:
        assert np.max(np.abs(r["chijj1_k"] - g["chijj1_k"])) <= TOL * s1
        assert np.max(np.abs(r["chijj2_k"] - g["chijj2_k"])) <= TOL * s2


@pytest.mark.parametrize("name", COND)
def test_chijj_matches_reference(name):
    g = load_golden(name)
    p = g["p"]
    c = _cond(p)
    c.solve()
    assert abs(c.scalars()["mu"] - g["s"]["mu"]) <= 1e-10 * max(1.0, abs(g["s"]["mu"]))
    r = c.calc_chijj_vertex_corr_all_optim(False, 3, _ntheta(g))
    _check(r, g)
    # the f-sum rule chi_jj(0) = -kx0 holds to the same accuracy as in the reference
    mine = (r["chijj1"][0] + r["chijj2"][0] + r["kx0"]) / r["kx0"]
    ref = (g["chijj1"][0] + g["chijj2"][0] + g["kx0"]) / g["kx0"]
    assert abs(mine - ref) <= 1e-9


def test_chijj_computes_sigma_and_mu_when_missing():
    """The reference runs calc_Self_FFT_spline, traceSelfG and find_mu itself
    when Sigma is missing (src/cond_opt.cpp:2550-2560)."""
    g = load_golden("l16_w128_n110")
    c = _cond(g["p"])
    r = c.calc_chijj_vertex_corr_all_optim()
    _check(r, g)


def test_chijj_repeat_is_bit_identical_and_bins_sum_to_totals():
    g = load_golden("l32_w256_u4_tp")
    c = _cond(g["p"])
    c.solve()
    a = c.calc_chijj_vertex_corr_all_optim(False, 3, 1)
    b = c.calc_chijj_vertex_corr_all_optim(False, 3, 5)
    d = c.calc_chijj_vertex_corr_all_optim(False, 3, 1)
    assert np.array_equal(a["chijj1"], d["chijj1"]) and np.array_equal(a["chijj2"], d["chijj2"])
    assert a["kx0"] == d["kx0"]
    for k in ("chijj1", "chijj2"):
        assert np.allclose(b[k + "_k"].sum(axis=1), a[k], rtol=0, atol=1e-14 * np.max(np.abs(a[k])))
        assert np.allclose(b[k], a[k], rtol=0, atol=1e-14 * np.max(np.abs(a[k])))


def test_chijj_bad_arguments():
    from tpsc_conductivity_b200 import _lib

    g = load_golden("l16_w64_u2")
    c = _cond(g["p"])
    with pytest.raises(_lib.TPSCError):
        c.ctx.call("tpsc_chijj", 1)  # no solve yet
    c.solve()
    with pytest.raises(_lib.TPSCError):
        c.ctx.call("tpsc_chijj", 0)


def test_sigma_iqn_is_the_kubo_form_of_chijj():
    g = load_golden("l128_w2048_cond")
    p = g["p"]
    c = _cond(p)
    c.solve()
    r = c.calc_chijj_vertex_corr_all_optim(False, 3, 1)
    s, sb = c.sigma_qn(256)
    qn = 2 * np.pi * np.arange(1, 257) * p["T"]
    assert np.allclose(s, (-r["kx0"] - r["chijj1"][1:257] - r["chijj2"][1:257]) / qn, rtol=1e-14, atol=0)
    assert np.allclose(sb, (-r["kx0"] - r["chijj1"][1:257]) / qn, rtol=1e-14, atol=0)
    # against the reference's chi_jj and kx0
    ref = (-float(g["kx0"]) - g["chijj1"][1:257] - g["chijj2"][1:257]) / qn
    scale = np.max(np.abs(g["chijj1"])) / qn
    assert np.all(np.abs(s - ref) <= 1e-10 * scale)


def test_pade_batch_reproduces_rational_functions():
    """A rational function with three poles is its own Pade approximant: the
    batched continuation recovers it on the real axis, and matches the oracle's
    restatement of generique::pade_cont_frac_coef_rec / pade."""
    from oracle import tpsc_oracle as O
    from tpsc_conductivity_b200.api import pade_batch

    T = 0.1
    poles = [np.array([0.3 - 0.2j, -1.1 - 0.5j, 2.0 - 0.1j]), np.array([0.7 - 0.3j, 1.5 - 0.05j, -0.4 - 1.0j])]
    res = [np.array([1.0, 0.5 + 0.2j, 0.25]), np.array([0.3, 0.1 - 0.1j, 2.0])]

    def f(k, z):
        return np.sum(res[k][:, None] / (z[None, :] - poles[k][:, None]), axis=0)

    z = np.linspace(0.0, 10.0, 2000) + 0.05j
    for Nn in (8, 16, 32):
        x = 1j * 2 * np.pi * np.arange(1, Nn + 1) * T
        y = np.stack([f(0, x), f(1, x)])
        out = pade_batch(x, y, z)
        for k in range(2):
            exact = f(k, z)
            assert np.max(np.abs(out[k] - exact)) <= 1e-9 * np.max(np.abs(exact)), (Nn, k)
            coef = O.pade_coefficients(y[k], x)
            ora = np.array([O.pade_eval(zz, x, coef) for zz in z[::50]])
            assert np.max(np.abs(out[k][::50] - ora)) <= 1e-9 * np.max(np.abs(ora)), (Nn, k)


def test_sigma_pade_interpolates_the_matsubara_data():
    from tpsc_conductivity_b200.api import pade_batch

    g = load_golden("l32_w256_u4_tp")
    p = g["p"]
    c = _cond(p)
    c.solve()
    c.calc_chijj_vertex_corr_all_optim()
    Nn = 64
    s, sb = c.sigma_qn(Nn)
    x = 1j * 2 * np.pi * np.arange(1, Nn + 1) * p["T"]
    back = pade_batch(x, np.stack([s, sb]).astype(complex), x)
    assert np.max(np.abs(back[0] - s) / np.abs(s)) <= 1e-11
    assert np.max(np.abs(back[1] - sb) / np.abs(sb)) <= 1e-11
    w = np.linspace(0.0, 10.0, 2000)
    sw, sbw = c.sigma_pade(w, Nn, 0.05)
    ref = pade_batch(x, np.stack([s, sb]).astype(complex), w + 0.05j)
    assert np.array_equal(sw, ref[0]) and np.array_equal(sbw, ref[1])
