"""The Newton-form solve queues chi0 -> roots -> vertex -> Sigma -> mu with no
host round trip (the root search takes its interval from the device chi0max,
the vertex and Sigma kernels read Usp, Uch from the device) and reads every
result back once at the end.  It must equal, bit for bit, the staged calls
that read each result back as they go, report a failed root search through
that one readback, and leave the context usable for the next solve."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

FORMS = ["newton", "mixed_newton"]


def _form(name):
    from tpsc_conductivity_b200 import _lib

    return _lib.FORM_NEWTON | (_lib.FORM_MIXED if name == "mixed_newton" else 0)


def _green(p, ctx, U=None):
    from tpsc_conductivity_b200.api import Green

    return Green(int(p["nk0"]), int(p["Nw0"]), p["n"], p["T"], 0.1,
                 (p["tp"], p["tpp"], p["t3"], p["U"] if U is None else U), ctx=ctx)


def _result(g):
    r = g.self_energy()
    return g.scalars(), r["S"].copy(), r["Sigma_inf2"].copy()


@pytest.mark.parametrize("form", FORMS)
def test_deferred_solve_equals_staged_calls(form):
    from tpsc_conductivity_b200.api import Context

    p = load_golden("l32_w256_u4_tp")["p"]
    ctx = Context(0)
    g = _green(p, ctx)
    g.set_form(_form(form))
    g.solve()
    s1, S1, a1 = _result(g)
    # the same stages, each read back before the next is queued
    g.calc_chiqw_FFT_spline()
    g.find_Usp_Uch_grid(int(p["nk0"]), int(p["Nw0"]))
    g.calc_chirt()
    g.calc_self_energy()
    g.find_mu()
    s2, S2, a2 = _result(g)
    assert np.array_equal(S1, S2) and np.array_equal(a1, a2)
    for k in ("Usp", "Uch", "mu", "chi0max", "Sigma_inf", "trSG2", "dblOcc"):
        if k in s1:
            assert s1[k] == s2[k], k


@pytest.mark.parametrize("form", FORMS)
def test_failed_root_search_is_reported_and_context_recovers(form):
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Context

    p = load_golden("l16_w128_n110")["p"]
    # the reference solve on a fresh context
    ref_ctx = Context(0)
    g0 = _green(p, ref_ctx)
    g0.set_form(_form(form))
    g0.solve()
    ref = _result(g0)
    # U = 5e-324 (the smallest positive double): the term Us nsr^2 / (2U) of
    # the spin sum rule overflows, so the device search stops at its first
    # evaluation without a root
    ctx = Context(0)
    bad = _green(p, ctx, U=5e-324)
    bad.set_form(_form(form))
    with pytest.raises(_lib.TPSCError, match="Usp not found"):
        bad.solve()
    # the same context solves the next point exactly as a fresh one does
    g = _green(p, ctx)
    g.set_form(_form(form))
    g.solve()
    got = _result(g)
    assert np.array_equal(got[1], ref[1]) and np.array_equal(got[2], ref[2])
    assert got[0] == ref[0]
