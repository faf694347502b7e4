"""The differentiation form: d(Usp, Uch, D)/d(U, mu, t') by forward tangents of
chi0 -> sum rules (tpsc_sumrule_tangents) against central finite differences
of the full-grid chi0 and sum-rule roots (h = 1e-5), FP64.

mu is a shift of the non-interacting chemical potential mu0 at fixed n
(tpsc_set_mu_shift), t' moves mu0 with the density held at n.  Tolerance:
1e-6 relative (+1e-9 absolute) -- the finite difference itself is good to
~1e-9 here (root tolerance 1e-16 over 2h, truncation h^2)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

H = 1e-5
CASES = {
    # the sensitivity workload: 128x128, U = 4, t' = -0.2, n = 0.85, T = 0.1, 1024 positive iwn
    "config4": dict(nk0=128, Nw0=2048, n=0.85, T=0.1, tp=-0.2, tpp=0.0, t3=0.0, U=4.0),
}
for nm in ("l32_w256_u4_tp", "l16_w128_n110"):
    p = load_golden(nm)["p"]
    CASES[nm] = dict(nk0=int(p["nk0"]), Nw0=int(p["Nw0"]), n=p["n"], T=p["T"], tp=p["tp"], tpp=p["tpp"],
                     t3=p["t3"], U=p["U"])


def _roots(c, form, dU=0.0, dmu=0.0, dtp=0.0):
    from tpsc_conductivity_b200.api import Green

    g = Green(c["nk0"], c["Nw0"], c["n"], c["T"], 0.1, (c["tp"] + dtp, c["tpp"], c["t3"], c["U"] + dU))
    g.set_form(form)
    g.set_mu_shift(dmu)
    Usp, Uch = g.find_Usp_Uch_grid(c["nk0"], c["Nw0"])
    n = c["n"]
    nsr = 2 - n if n > 1 else n
    D = Usp / (c["U"] + dU) * nsr * nsr / 4.0 + (1 - nsr if n > 1 else 0.0)
    return np.array([Usp, Uch, D]), g


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("form_name", ["reference", "newton"])
def test_tangents_match_central_differences(name, form_name):
    from tpsc_conductivity_b200 import _lib

    form = _lib.FORM_NEWTON if form_name == "newton" else _lib.FORM_REFERENCE
    c = CASES[name]
    base, g = _roots(c, form)
    J = g.sumrule_tangents()
    fd = {
        "U": (_roots(c, form, dU=H)[0] - _roots(c, form, dU=-H)[0]) / (2 * H),
        "mu": (_roots(c, form, dmu=H)[0] - _roots(c, form, dmu=-H)[0]) / (2 * H),
        "tp": (_roots(c, form, dtp=H)[0] - _roots(c, form, dtp=-H)[0]) / (2 * H),
    }
    report = {}
    for p, f in fd.items():
        for k, v in zip(("Usp", "Uch", "D"), f):
            report[p + "/" + k] = (J[p][k], v)
            assert abs(J[p][k] - v) <= 1e-6 * abs(v) + 1e-9, (p, k, J[p][k], v)
    print(name, form_name, {k: "%.9g vs %.9g" % t for k, t in report.items()})
    # the backward pair is the transpose product of the same Jacobian
    cot = np.array([0.3, -1.2, 2.5])
    grad = g.sumrule_vjp(cot)
    for i, p in enumerate(("U", "mu", "tp")):
        ref = cot[0] * J[p]["Usp"] + cot[1] * J[p]["Uch"] + cot[2] * J[p]["D"]
        assert abs(grad[i] - ref) <= 1e-12 * max(1.0, abs(ref))


def test_tangents_need_the_roots():
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Green

    c = CASES["l16_w128_n110"]
    g = Green(c["nk0"], c["Nw0"], c["n"], c["T"], 0.1, (c["tp"], c["tpp"], c["t3"], c["U"]))
    with pytest.raises(_lib.TPSCError):
        g.sumrule_tangents()
    g.calc_chiqw_FFT_spline()
    with pytest.raises(_lib.TPSCError):
        g.sumrule_tangents()
