"""The reverse pass of sigma(iq_n) (tpsc_sigma_iqn_bwd): V -> Sigma -> mu ->
chi_jj -> sigma backward on the device, chained with the forward tangents of
chi0 and of the sum-rule roots, against central differences of full FP64
device solves (tpsc_sigma_iqn_fd) and of the oracle's forward.

* 16 x 16, 64 frequencies: the gradient of sigma(iq_1) against central
  differences (h = 1e-5) of the oracle's own solve + conductivity (numpy,
  run here): 1e-7 relative.
* 32 x 32 and the adjoint workload's 128 x 128, 1024 positive frequencies
  (U = 4, t' = -0.2, n = 0.85, T = 0.1): the gradient of sigma(iq_1), and of
  a random combination of sigma(iq_1..4), against the device's central
  differences: 1e-6 relative to the largest component (the differences carry
  O(h^2) truncation and the roots' convergence error / h).
* dD equals the sum-rule tangents'; bad arguments are rejected.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ADJ = dict(nk0=128, Nw0=2048, n=0.85, T=0.1, tp=-0.2, U=4.0)


def _cond_green(m, form=None):
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import CondOpt

    g = CondOpt(m["nk0"], m["Nw0"], m["n"], m["T"], 0.1, (m["tp"], 0.0, 0.0, m["U"]))
    g.set_form(_lib.FORM_NEWTON if form is None else form)
    g.solve()
    g.ctx.call("tpsc_chijj", 1)
    g._nbins = 1
    return g


@pytest.mark.parametrize("m", [dict(nk0=32, Nw0=256, n=0.85, T=0.1, tp=-0.2, U=4.0), ADJ],
                         ids=["l32_w256", "l128_w2048"])
def test_reverse_pass_matches_device_central_differences(m):
    g = _cond_green(m)
    nq = 4
    ds, dD_fd = g.sigma_qn_sensitivities(nq)           # [3, nq]; re-solves the base point
    g.ctx.call("tpsc_chijj", 1)
    grad1, dD = g.sigma_qn_vjp([1.0])
    scale = np.max(np.abs(ds[:, 0]))
    err1 = np.max(np.abs(grad1 - ds[:, 0])) / scale
    rng = np.random.default_rng(7)
    cot = rng.standard_normal(nq)
    gradc, _ = g.sigma_qn_vjp(cot)
    ref = ds @ cot
    errc = np.max(np.abs(gradc - ref)) / np.max(np.abs(ref))
    print(f"{m['nk0']}^2 x {m['Nw0']}: reverse pass {grad1}, differences {ds[:, 0]}, "
          f"rel err {err1:.2e}; 4-frequency cotangent rel err {errc:.2e}")
    assert err1 < 1e-6
    assert errc < 1e-6
    J = g.sumrule_tangents()
    for i, p in enumerate(("U", "mu", "tp")):
        assert dD[i] == pytest.approx(J[p]["D"], rel=1e-12, abs=1e-15)


def test_reverse_pass_matches_the_oracle_forward():
    from oracle import tpsc_oracle as O

    m = dict(nk0=16, Nw0=64, n=0.87, T=0.25, tp=-0.15, U=2.5)
    g = _cond_green(m)
    grad, _ = g.sigma_qn_vjp([1.0])

    def sig1(U, tp, dmu):
        nbk = m["nk0"] // 2 + 1
        ek = O.dispersion(nbk, tp, 0.0, 0.0)
        er = O.hopping_octant(nbk, tp, 0.0, 0.0)
        mu0 = O.mu0_finite(ek, m["n"], m["T"], tp, 0.0) + dmu
        c0 = O.chi0_fft_spline(ek, mu0, m["T"], er, m["Nw0"])
        ur = O.find_Usp_Uch(c0, U, m["n"], m["T"])
        V = O.vertex_rt(c0, U, ur.Usp, ur.Uch, m["T"])
        sr = O.self_energy(ek, mu0, m["T"], er, c0, V, U, ur.Usp, ur.Uch, m["Nw0"])
        mu, _ = O.find_mu(ek, mu0, sr, m["T"])
        sv = O.Solve(m["nk0"], m["Nw0"], mu0, c0, ur, V, sr, mu, None, None)
        cr = O.conductivity(sv, tp, 0.0, 0.0, U, m["T"])
        q1 = 2 * np.pi * m["T"]
        return (-cr.kx0 - cr.chijj1[1] - cr.chijj2[1]) / q1

    h = 1e-5
    U, tp = m["U"], m["tp"]
    fd = np.array([(sig1(U + h, tp, 0.0) - sig1(U - h, tp, 0.0)) / (2 * h),
                   (sig1(U, tp, h) - sig1(U, tp, -h)) / (2 * h),
                   (sig1(U, tp + h, 0.0) - sig1(U, tp - h, 0.0)) / (2 * h)])
    err = np.max(np.abs(grad - fd)) / np.max(np.abs(fd))
    print(f"16^2 x 64: reverse pass {grad}, oracle differences {fd}, rel err {err:.2e}")
    assert err < 1e-7


def test_mixed_form_point_gives_the_gradient_within_its_bound():
    from tpsc_conductivity_b200 import _lib

    m = dict(nk0=32, Nw0=256, n=0.85, T=0.1, tp=-0.2, U=4.0)
    g64 = _cond_green(m)
    ref, _ = g64.sigma_qn_vjp([1.0])
    g32 = _cond_green(m, _lib.FORM_NEWTON | _lib.FORM_MIXED)
    got, _ = g32.sigma_qn_vjp([1.0])
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref))


def test_bad_arguments_are_rejected():
    from tpsc_conductivity_b200 import _lib

    m = dict(nk0=16, Nw0=64, n=0.87, T=0.25, tp=-0.15, U=2.5)
    g = _cond_green(m)
    for cot in ([], np.ones(33), [np.nan]):
        with pytest.raises(_lib.TPSCError) as e:
            g.sigma_qn_vjp(cot)
        assert e.value.status == _lib.ERR_ARG
