"""Sensitivities of sigma(iq_n) and of the double occupancy to U, mu and t'
(tpsc_sigma_iqn_fd: central differences of full FP64 device solves), on the
adjoint workload's model: 128x128 lattice, U = 4, t' = -0.2, n = 0.85,
T = 0.1, 1024 positive fermionic frequencies.

* dD/d(U, mu, t') agrees with the forward tangents of the sum-rule stage
  (tpsc_sumrule_tangents) to 1e-5 relative: the central difference with
  h = 1e-5 carries O(h^2) truncation and the roots' convergence error / h.
* d sigma(iq_n)/d theta is stable under the step: h = 1e-5 and 2e-5 agree
  to 1e-6 of the largest derivative.
* The context is left at its own parameters: the scalars and sigma(iq_n)
  after the call are those of a plain solve."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODEL = dict(nk0=128, Nw0=2048, n=0.85, T=0.1, tp=-0.2, U=4.0)
NQ = 4


def _green():
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import CondOpt

    m = MODEL
    g = CondOpt(m["nk0"], m["Nw0"], m["n"], m["T"], 0.1, (m["tp"], 0.0, 0.0, m["U"]))
    g.set_form(_lib.FORM_NEWTON)
    return g


def _base(g):
    g.solve()
    g.ctx.call("tpsc_chijj", 1)
    g._nbins = 1
    return g.scalars(), g.sigma_qn(NQ)[0]


def test_dD_matches_the_sumrule_tangents():
    g = _green()
    _base(g)
    ds, dD = g.sigma_qn_sensitivities(NQ)
    J = g.sumrule_tangents()
    for i, p in enumerate(("U", "mu", "tp")):
        ref = J[p]["D"]
        assert abs(dD[i] - ref) <= 1e-5 * max(abs(ref), 1e-3), (p, dD[i], ref)
    assert np.all(np.isfinite(ds))
    assert np.max(np.abs(ds)) > 0


def test_sigma_derivative_is_stable_under_the_step():
    g = _green()
    _base(g)
    d1, _ = g.sigma_qn_sensitivities(NQ, h=(1e-5, 1e-5, 1e-5))
    d2, _ = g.sigma_qn_sensitivities(NQ, h=(2e-5, 2e-5, 2e-5))
    for p in range(3):
        scale = np.max(np.abs(d1[p]))
        assert scale > 0
        assert np.max(np.abs(d1[p] - d2[p])) <= 1e-6 * scale, p


def test_context_is_left_at_its_own_parameters():
    g = _green()
    s0, sig0 = _base(g)
    g.sigma_qn_sensitivities(NQ)
    s1 = g.scalars()
    sig1 = g.sigma_qn(NQ)[0]
    for k in ("Usp", "Uch", "mu", "mu0", "Sigma_inf"):
        assert abs(s1[k] - s0[k]) <= 1e-12 * max(1.0, abs(s0[k])), k
    assert np.max(np.abs(sig1 - sig0)) <= 1e-12 * np.max(np.abs(sig0))


def test_bad_steps_are_rejected():
    from tpsc_conductivity_b200 import _lib

    g = _green()
    _base(g)
    for kw in (dict(nq=NQ, h=(1e-5, 0.0, 1e-5)), dict(nq=0), dict(nq=MODEL["Nw0"] // 2 + 1)):
        with pytest.raises(_lib.TPSCError) as e:
            g.sigma_qn_sensitivities(**kw)
        assert e.value.status == _lib.ERR_ARG
