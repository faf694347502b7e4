"""Tilings of the tau transforms (tpsc_tune_tau_tiles / tpsc_set_tau_tile):
one column pair per CTA and four columns per CTA compute the same spline +
FFT, so a solve with either tiling gives the same results (1e-11), and the
tuner's choice leaves a re-solve unchanged.  The tiling is process-wide; every
test puts the default (pairs) back."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(16, 64), (32, 256), (64, 2048), (32, 4096)]
MODEL = dict(n=0.875, T=0.1, tp=-0.15, U=3.0)


def _solve(nk0, Nw0, form):
    from tpsc_conductivity_b200.api import Green

    g = Green(nk0, Nw0, MODEL["n"], MODEL["T"], 0.1, (MODEL["tp"], 0.0, 0.0, MODEL["U"]))
    g.set_form(form)
    g.solve()
    return g, g.scalars(), g.sigma()


def _set_all(lib, Nw0, tile):
    for kind in range(3):
        assert lib.tpsc_set_tau_tile(kind, Nw0, tile) == 0


def _close(a, b):
    sa, Sa = a
    sb, Sb = b
    assert np.max(np.abs(Sa - Sb)) <= 1e-11 * np.max(np.abs(Sb))
    for k in ("Usp", "Uch", "mu", "chi0max", "Sigma_inf"):
        assert abs(sa[k] - sb[k]) <= 1e-11 * max(1.0, abs(sb[k])), k


@pytest.mark.parametrize("nk0,Nw0", SHAPES)
def test_both_tilings_give_the_same_solve(nk0, Nw0):
    from tpsc_conductivity_b200 import _lib

    lib = _lib.load()
    form = _lib.FORM_NEWTON
    try:
        _set_all(lib, Nw0, 0)
        _, s0, S0 = _solve(nk0, Nw0, form)
        _set_all(lib, Nw0, 1)
        _, s1, S1 = _solve(nk0, Nw0, form)
        _close((s1, S1), (s0, S0))
    finally:
        _set_all(lib, Nw0, 0)


def test_tuner_times_both_and_keeps_the_results():
    from tpsc_conductivity_b200 import _lib

    lib = _lib.load()
    nk0, Nw0 = 64, 2048
    try:
        g, s0, S0 = _solve(nk0, Nw0, _lib.FORM_NEWTON | _lib.FORM_MIXED)
        ms = np.zeros(6)
        assert lib.tpsc_tune_tau_tiles(g.ctx.h, 3, ms.ctypes.data_as(C.POINTER(C.c_double))) == 0
        assert np.all(ms > 0)
        # the stages are stale after tuning; a solve recomputes them
        g.solve()
        _close((g.scalars(), g.sigma()), (s0, S0))
        assert lib.tpsc_set_tau_tile(3, Nw0, 0) == _lib.ERR_ARG
    finally:
        _set_all(lib, Nw0, 0)


@pytest.mark.parametrize("nk0,Nw0", [(16, 64), (32, 256), (64, 2048)])
def test_radix8_plan_gives_the_same_solve(nk0, Nw0):
    """Plan 2: one column pair per CTA with radix-8 FFT passes (twice the
    threads in each FFT) -- the same spline + FFT as plan 0."""
    from tpsc_conductivity_b200 import _lib

    lib = _lib.load()
    form = _lib.FORM_NEWTON | _lib.FORM_MIXED
    try:
        _set_all(lib, Nw0, 0)
        _, s0, S0 = _solve(nk0, Nw0, form)
        _set_all(lib, Nw0, 2)
        _, s2, S2 = _solve(nk0, Nw0, form)
        _close((s2, S2), (s0, S0))
    finally:
        _set_all(lib, Nw0, 0)


def test_plan_tuner_times_three_plans_and_keeps_the_results():
    from tpsc_conductivity_b200 import _lib

    lib = _lib.load()
    nk0, Nw0 = 64, 1024
    try:
        g, s0, S0 = _solve(nk0, Nw0, _lib.FORM_NEWTON | _lib.FORM_MIXED)
        ms = np.zeros(9)
        assert lib.tpsc_tune_tau_plans(g.ctx.h, 3, ms.ctypes.data_as(C.POINTER(C.c_double))) == 0
        assert np.all(ms > 0), ms
        print("tau plans (chi0, V, Sigma) x (pair r16, four columns, pair r8) ms:", np.round(ms.reshape(3, 3), 4))
        g.solve()
        _close((g.scalars(), g.sigma()), (s0, S0))
        # plan 2 needs Nw0 <= 2048
        assert lib.tpsc_set_tau_tile(0, 4096, 2) == _lib.ERR_ARG
    finally:
        _set_all(lib, Nw0, 0)
