"""Pin the numpy oracle to the reference: every golden fixture was produced by
the unmodified reference sources (tests/golden/make_golden.py); the oracle must
reproduce them.  Tolerances are relative to the array's max magnitude; the
reference's own run-to-run noise (OpenMP reduction order) is ~1e-12 on Usp,
Uch and mu at L=256."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from oracle import tpsc_oracle as O

SMALL = [n for n in golden_names() if not n.startswith(("l256", "l128"))]


def full_sigma(g, S, T, cols=None):
    """Sigma(k, iw_n) = Sigma_inf/z + C2/z^2 + C3/z^3 + S/z^4 (src/green.cpp:3039)."""
    s2, s3 = g["sigma_inf2"], g["sigma_inf3"]
    if cols is not None:
        s2, s3 = s2[cols], s3[cols]
    z = 1j * (2 * np.arange(S.shape[0])[:, None] + 1) * np.pi * T
    return g["s"]["Sigma_inf"] / z + s2 / z ** 2 + s3 / z ** 3 + S / z ** 4


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", SMALL)
def test_oracle_matches_reference(name):
    g = load_golden(name)
    p, s = g["p"], g["s"]
    r = O.solve(p["U"], p["tp"], p["tpp"], p["t3"], p["n"], p["T"], p["nk0"], p["Nw0"])
    assert abs(r.mu0 - s["mu0"]) <= 1e-12 * max(1.0, abs(s["mu0"]))
    assert r.chi0.qmax == (int(s["qmax0"]), int(s["qmax1"]))
    assert rel(r.chi0.chi0max, s["chi0max"]) < 1e-12
    assert rel(r.chi0.chi0_inf, g["chi0_inf"]) < 1e-12
    # Nyquist component of the spline third derivative: an alternating sum, so
    # two exact spline solvers differ here at ~1e-9 of the max (it only weights
    # the 1/qn^4 tail beyond the stored frequencies)
    assert rel(r.chi0.chi0_inf2, g["chi0_inf2"]) < 1e-8
    assert rel(r.chi0.dtau_chirt0, g["dtau_chirt0"]) < 1e-12
    if "chiqw" in g:
        assert rel(r.chi0.chiqw, g["chiqw"]) < 1e-11
        assert rel(r.V, g["vertex_rt"]) < 1e-11
        # S multiplies 1/z^4: its high-frequency end is an alternating sum of
        # spline third derivatives and carries ~1e-9 (of max) solver noise
        assert rel(r.sigma.S, g["self"]) < 1e-8
        assert rel(r.sigma.sigma(p["T"]), full_sigma(g, g["self"], p["T"])) < 1e-11
    else:
        c = g["cols"]
        assert rel(r.chi0.chiqw[:, c], g["chiqw_cols"]) < 1e-11
        assert rel(r.chi0.chiqw[0], g["chiqw_w0"]) < 1e-11
        assert rel(r.V[:, c], g["vertex_rt_cols"]) < 1e-11
        assert rel(r.sigma.S[:, c], g["self_cols"]) < 1e-8
        # two runs of the reference binary itself differ by ~1e-11 (of max) in
        # the full Sigma on these columns at 64^2 x 1024 (OpenMP reduction order)
        assert rel(r.sigma.sigma(p["T"])[:, c], full_sigma(g, g["self_cols"], p["T"], c)) < 3e-11
    assert rel(r.U.Usp, s["Usp"]) < 1e-10
    assert rel(r.U.Uch, s["Uch"]) < 1e-10
    assert rel(r.U.dblOcc, s["dblOcc"]) < 1e-10
    assert rel(r.sigma.Sigma_inf, s["Sigma_inf"]) < 1e-10
    assert rel(r.sigma.Sigma_inf2, g["sigma_inf2"]) < 1e-10
    assert rel(r.sigma.Sigma_inf3, g["sigma_inf3"]) < 1e-9
    assert rel(r.sigma.Sigma_inf4, g["sigma_inf4"]) < 1e-8
    assert abs(r.mu - s["mu"]) < 1e-10 * max(1.0, abs(s["mu"]))


def test_spline_matches_definition():
    """The M-form clamped spline interpolates, is C2 and has the end slopes."""
    rng = np.random.default_rng(1)
    V = rng.standard_normal((33, 3))
    h = 0.1
    d0, dN = rng.standard_normal(3), rng.standard_normal(3)
    a, b, c, d = O.clamped_spline(V, h, d0, dN)
    assert np.allclose(a * h ** 3 + b * h * h + c * h + d, V[1:], atol=1e-12)
    assert np.allclose(3 * a[:-1] * h * h + 2 * b[:-1] * h + c[:-1], c[1:], atol=1e-11)
    assert np.allclose(6 * a[:-1] * h + 2 * b[:-1], 2 * b[1:], atol=1e-9)
    assert np.allclose(c[0], d0)
    assert np.allclose(3 * a[-1] * h * h + 2 * b[-1] * h + c[-1], dN, atol=1e-11)


def test_find_zero_quadratic():
    root, nev = O.find_zero(lambda x: x * x - 2.0, (1.0, 0.0, 3.0))
    assert abs(root - np.sqrt(2.0)) < 1e-15
    root, nev = O.find_zero(lambda x: x - 0.3, (0.0, -10.0, 10.0), lims=(-20, 20))
    assert abs(root - 0.3) < 1e-15


CONT = [n for n in SMALL if "mdc_A" in load_golden(n)]


def check_fs(mine, ref):
    """Rows (l + m*, m*, A*) of find_FS_inter.  The maxima must agree; the
    arg-max may differ only where the line has two equal maxima (symmetric
    points about a particle-hole symmetric Fermi surface), where rounding
    decides."""
    assert np.allclose(mine[:, 2], ref[:, 2], rtol=1e-6)
    for a, b in zip(mine, ref):
        if a[1] != b[1]:
            assert abs(a[2] - b[2]) <= 1e-6 * abs(b[2])


@pytest.mark.parametrize("name", CONT)
def test_oracle_continuation_matches_reference(name):
    """MDC (10-point Pade at w = 0, 4 etas), find_FS_inter and Gwn_local against
    the reference's own text output (written with 8-12 significant digits)."""
    g = load_golden(name)
    p = g["p"]
    r = O.solve(p["U"], p["tp"], p["tpp"], p["t3"], p["n"], p["T"], p["nk0"], p["Nw0"])
    ek = O.dispersion(p["nk0"] // 2 + 1, p["tp"], p["tpp"], p["t3"])
    etas = np.array([0.01, 0.001, 0.0001, 0.00001])
    s, A = O.pade_sigma(ek, r.mu, r.sigma, p["T"], 1j * etas, np.arange(10), 10, mode=0)
    assert np.allclose(A, g["mdc_A"], rtol=1e-6, atol=1e-11)
    assert np.allclose(s, g["mdc_sigma"], rtol=1e-6, atol=1e-11)
    poly, pade = O.fs_inter(ek, r.mu, r.sigma, p["T"])
    check_fs(poly, g["fs_inter"])
    check_fs(pade, g["fs_inter_pade"])
    assert np.allclose(O.gwn_local(ek, r.mu, r.sigma, p["T"]), g["gwn_local"], rtol=1e-8, atol=1e-11)


@pytest.mark.parametrize("name,ntheta", [(n, 1) for n in CONT] + [("l32_w256_theta3", 3)])
def test_oracle_conductivity_matches_reference(name, ntheta):
    """Bubble chi_jj, the Maki-Thompson correction, kx0 and the angle-resolved
    sums (cond_opt::calc_chijj_vertex_corr_all_optim, src/cond_opt.cpp:2537-4286)
    against the reference's own arrays."""
    g = load_golden(name)
    p = g["p"]
    r = O.solve(p["U"], p["tp"], p["tpp"], p["t3"], p["n"], p["T"], p["nk0"], p["Nw0"])
    c = O.conductivity(r, p["tp"], p["tpp"], p["t3"], p["U"], p["T"], ntheta)
    scale1 = np.max(np.abs(g["chijj1"]))
    scale2 = np.max(np.abs(g["chijj2"]))
    assert np.max(np.abs(c.chijj1 - g["chijj1"])) <= 1e-11 * scale1
    assert np.max(np.abs(c.chijj2 - g["chijj2"])) <= 1e-11 * scale2
    assert abs(c.kx0 - float(g["kx0"])) <= 1e-12 * abs(float(g["kx0"]))
    if ntheta > 1:
        assert np.max(np.abs(c.chijj1_k - g["chijj1_k"])) <= 1e-11 * scale1
        assert np.max(np.abs(c.chijj2_k - g["chijj2_k"])) <= 1e-11 * scale2


@pytest.mark.parametrize("name", golden_names())
def test_oracle_sp_corr_length_matches_reference(name):
    """chi::sp_corr_length (src/chi.cpp:450-718) with vF at the hot spots of
    green0::find_FS(10001) (src/green0.cpp:626-676), restated, on the
    reference's own chi0(q, 0), chi0max, qmax, Usp and mu0 -- commensurate and
    incommensurate (l64, l256) peaks, n > 1, half filling."""
    g = load_golden(name)
    p, s = g["p"], g["s"]
    q0 = g["chiqw"][0] if "chiqw" in g else g["chiqw_w0"]
    r = O.sp_corr_length(q0, s["chi0max"], (int(s["qmax0"]), int(s["qmax1"])), s["Usp"], int(p["nk0"]) // 2 + 1,
                         s["mu0"], p["tp"], p["tpp"], p["t3"])
    for k, v in zip(g["corr_names"], g["corr"]):
        assert abs(r[str(k)] - v) <= 1e-13 * abs(v), (k, r[str(k)], v)


AL = [n for n in golden_names() if n.startswith("al_")]


@pytest.mark.parametrize("name", AL)
def test_oracle_al_matches_reference(name):
    """The Aslamazov-Larkin correction chijj3 on the non-uniform iqn grid
    (cond_opt::calc_chijj_vertex_corr_all_optim with chi3 = true,
    src/cond_opt.cpp:4292-6529) against the reference's own array: mmin 2, 3
    and 4, n < 1, n = 1 and n > 1, angle bins."""
    g = load_golden(name)
    p = g["p"]
    ntheta = g["chijj3_k"].shape[1] if "chijj3_k" in g else 1
    r = O.solve(p["U"], p["tp"], p["tpp"], p["t3"], p["n"], p["T"], p["nk0"], p["Nw0"])
    a = O.conductivity_al(r, p["tp"], p["tpp"], p["t3"], p["U"], p["T"], int(g["mmin"]), ntheta)
    assert np.array_equal(a.ind_freq, g["ind_freq"])
    scale = np.max(np.abs(g["chijj3"]))
    assert np.max(np.abs(a.chijj3 - g["chijj3"])) <= 1e-10 * scale
    if ntheta > 1:
        assert np.max(np.abs(a.chijj3_k[1:] - g["chijj3_k"])) <= 1e-10 * scale
