"""The mixed-precision form (FP32 G, chi0, V and Sigma slice transforms with
compensated twiddles, the Sigma slice's local term in FP64; everything else
FP64) against the FP64 form on the same inputs: the error of every output,
with the bound each must meet, at every size up to 256 x 256 with 2048
positive Matsubara frequencies.

  Sigma(k, i w_n) (full), sigma(iq_n) with vertex correction   <= 1e-6 of max |.|
  chi0(q, iqn), V(r, tau)                                       <= 1e-6 of max |.|
  Usp, Uch, double occupancy, mu, Sigma_inf                     <= 1e-6 relative

Each case prints its measured errors (run pytest with -s to see them).
"""
import json

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

CASES = ["l32_w256_u4_tp", "l16_w128_n110", "l32_w512_u2", "l128_w2048_cond", "l256_w4096_u4"]
TOL = 1e-6


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def _solve(p, form):
    from tpsc_conductivity_b200.api import CondOpt

    c = CondOpt(p["nk0"], p["Nw0"], p["n"], p["T"], 0.1, (p["tp"], p["tpp"], p["t3"], p["U"]))
    c.set_form(form)
    c.solve()
    out = {"s": c.scalars(), "sigma": c.sigma(), "chi0": c.chi0()["chiqw"], "V": c.vertex()}
    c.calc_chijj_vertex_corr_all_optim(False, 3, 1)
    nq = min(256, p["Nw0"] // 2)
    out["sig_qn"] = c.sigma_qn(nq)[0]
    return out


@pytest.mark.parametrize("name", CASES)
def test_mixed_form_error_against_fp64(name):
    from tpsc_conductivity_b200 import _lib

    g = load_golden(name)
    p = g["p"]
    ref = _solve(p, _lib.FORM_NEWTON)
    mix = _solve(p, _lib.FORM_NEWTON | _lib.FORM_MIXED)
    err = {
        "Sigma": rel(mix["sigma"], ref["sigma"]),
        "chi0": rel(mix["chi0"], ref["chi0"]),
        "V": rel(mix["V"], ref["V"]),
    }
    for k in ("Usp", "Uch", "dblOcc", "mu", "Sigma_inf"):
        err[k] = abs(mix["s"][k] - ref["s"][k]) / max(abs(ref["s"][k]), 1e-12)
    err["sigma_qn"] = rel(mix["sig_qn"], ref["sig_qn"])
    print("mixed-form error", name, json.dumps({k: float("%.3g" % v) for k, v in err.items()}))
    for k, v in err.items():
        assert v <= TOL, (k, v)
    # and the FP64 Newton form against the reference's own scalars
    s = g["s"]
    assert abs(ref["s"]["Usp"] - s["Usp"]) <= 1e-9 * s["Usp"]
