"""The plans of the mixed form's FP32 slice transforms (tpsc_set_slice_plan):
packed radix-16 FFTs of the even extension (plan 0), the folded matrix
DCT-I on the FP32 pipe (plan 1) and, for the V and Sigma slices of the
256 x 256 lattice, the same matrix DCT-I on the tcgen05 tensor cores in
3xTF32 (plan 2).  All compute the reference's REDFT00 x REDFT00 of the same slices, so a
mixed + Newton solve with any plan is within the mixed form's bound of the
FP64 Newton solve (Sigma, chi0, V and the scalars to 1e-6), and the plans
agree with each other to the same bound.  Settings are process-wide; every
test puts the defaults back.
"""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (nk0, Nw0, n, T, t', U)
SHAPES = [(64, 1024, 0.875, 0.1, -0.15, 3.0), (128, 2048, 0.9, 0.1, 0.0, 3.0), (256, 4096, 0.875, 0.05, -0.15, 4.0)]
TOL = 1e-6


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def _solve(shape, form):
    from tpsc_conductivity_b200.api import Green

    nk0, Nw0, n, T, tp, U = shape
    g = Green(nk0, Nw0, n, T, 0.1, (tp, 0.0, 0.0, U))
    g.set_form(form)
    g.solve()
    out = {"s": g.scalars(), "sigma": g.sigma(), "chi0": g.chi0()["chiqw"], "V": g.vertex()}
    g.ctx.close()
    return out


def _errors(a, ref):
    err = {k: rel(a[k], ref[k]) for k in ("sigma", "chi0", "V")}
    for k in ("Usp", "Uch", "mu", "Sigma_inf"):
        err[k] = abs(a["s"][k] - ref["s"][k]) / max(abs(ref["s"][k]), 1e-12)
    return err


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"l{s[0]}_w{s[1]}")
def test_plans_agree_within_the_mixed_bound(shape):
    from tpsc_conductivity_b200 import _lib

    lib = _lib.load()
    nk0 = shape[0]
    defaults = [lib.tpsc_get_slice_plan(k, nk0) for k in range(4)]
    ref = _solve(shape, _lib.FORM_NEWTON)
    out = {}
    try:
        for plan in (0, 1):
            for kind in range(4):
                assert lib.tpsc_set_slice_plan(kind, nk0, plan) == 0
            out[plan] = _solve(shape, _lib.FORM_NEWTON | _lib.FORM_MIXED)
    finally:
        for kind in range(4):
            assert lib.tpsc_set_slice_plan(kind, nk0, defaults[kind]) == 0
    errs = {plan: _errors(out[plan], ref) for plan in (0, 1)}
    between = _errors(out[1], out[0])
    print("slice plans", nk0, json.dumps({str(k): {a: float("%.3g" % b) for a, b in v.items()}
                                         for k, v in {**errs, "1v0": between}.items()}))
    for plan in (0, 1):
        for k, v in errs[plan].items():
            assert v <= TOL, (plan, k, v)
    for k, v in between.items():
        assert v <= TOL, ("between", k, v)


@pytest.mark.parametrize("kinds", [(3,), (2, 3)], ids=["sigma", "vertex_sigma"])
@pytest.mark.parametrize("nw0", [512, 4096])
def test_tensor_plan(nw0, kinds):
    """Plan 2 (tensor cores) for the Sigma slice alone and for the V and
    Sigma slices, against plan 0 and the FP64 solve, with the tensor plan's
    error word checked clear."""
    import ctypes as C

    from tpsc_conductivity_b200 import _lib

    lib = _lib.load()
    shape = (256, nw0, 0.875, 0.05, -0.15, 4.0)
    defaults = [lib.tpsc_get_slice_plan(k, 256) for k in range(4)]
    word = C.c_uint(0)
    assert lib.tpsc_tensor_plan_errors(C.byref(word), 1) == 0
    ref = _solve(shape, _lib.FORM_NEWTON)
    out = {}
    try:
        for plan in (0, 2):
            for kind in range(4):
                assert lib.tpsc_set_slice_plan(kind, 256, plan if kind in kinds else 0) == 0
            out[plan] = _solve(shape, _lib.FORM_NEWTON | _lib.FORM_MIXED)
    finally:
        for kind in range(4):
            assert lib.tpsc_set_slice_plan(kind, 256, defaults[kind]) == 0
    assert lib.tpsc_tensor_plan_errors(C.byref(word), 1) == 0
    assert word.value == 0
    errs = {plan: _errors(out[plan], ref) for plan in (0, 2)}
    between = _errors(out[2], out[0])
    print("tensor plan", nw0, kinds, json.dumps({str(k): {a: float("%.3g" % b) for a, b in v.items()}
                                         for k, v in {**errs, "2v0": between}.items()}))
    for plan in (0, 2):
        for k, v in errs[plan].items():
            assert v <= TOL, (plan, k, v)
    for k, v in between.items():
        assert v <= TOL, ("between", k, v)


def test_slice_plan_tuner_keeps_the_fastest_and_the_results():
    """tpsc_tune_slice_plans times every plan of each slice kind after a
    mixed-form solve, keeps the fastest, and a re-solve with the chosen plans
    stays within the mixed form's bound of the FP64 solve."""
    import ctypes as C

    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Green

    lib = _lib.load()
    shape = (256, 1024, 0.875, 0.1, -0.15, 3.0)
    nk0 = shape[0]
    defaults = [lib.tpsc_get_slice_plan(k, nk0) for k in range(4)]
    ref = _solve(shape, _lib.FORM_NEWTON)
    try:
        nk0_, Nw0, n, T, tp, U = shape
        g = Green(nk0_, Nw0, n, T, 0.1, (tp, 0.0, 0.0, U))
        g.set_form(_lib.FORM_NEWTON | _lib.FORM_MIXED)
        g.solve()
        ms = np.zeros(12)
        assert lib.tpsc_tune_slice_plans(g.ctx.h, 3, ms.ctypes.data_as(C.POINTER(C.c_double))) == 0
        print("slice plan times (ms, [kind][plan])", ms.reshape(4, 3).round(4).tolist())
        for kind in range(4):
            t = ms[3 * kind:3 * kind + 3]
            chosen = lib.tpsc_get_slice_plan(kind, nk0)
            assert t[chosen] > 0 and t[chosen] == min(x for x in t if x > 0), (kind, t, chosen)
        g.solve()
        out = {"s": g.scalars(), "sigma": g.sigma(), "chi0": g.chi0()["chiqw"], "V": g.vertex()}
        g.ctx.close()
    finally:
        for kind in range(4):
            assert lib.tpsc_set_slice_plan(kind, nk0, defaults[kind]) == 0
    for k, v in _errors(out, ref).items():
        assert v <= TOL, (k, v)


def test_tensor_plan_in_batched_points():
    """The tensor plan's kernels over the points of a batched launch (one
    launch per stage over every point of a shape group, the TMA tensor maps
    spanning the points' arenas) give each point's one-point solve with the
    same plans to 1e-11."""
    import ctypes as C

    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Context, Green

    lib = _lib.load()
    defaults = [lib.tpsc_get_slice_plan(k, 256) for k in range(4)]
    P = np.array([[256, 512, 0.875, 0.05, -0.15, 0.0, 0.0, 4.0],
                  [256, 512, 0.9, 0.08, -0.1, 0.0, 0.0, 3.0],
                  [256, 512, 0.8, 0.06, -0.2, 0.0, 0.0, 5.0]], dtype=np.float64)
    names = list(_lib.SCALARS)
    try:
        for kind in range(4):
            assert lib.tpsc_set_slice_plan(kind, 256, 2 if kind >= 2 else 0) == 0
        ctx = Context()
        n = P.shape[0]
        res = np.zeros((n, len(names)))
        st = np.zeros(n, dtype=np.int32)
        ms = np.zeros(1)
        ctx.call("tpsc_solve_points", n, P.ctypes.data_as(C.POINTER(C.c_double)),
                 res.ctypes.data_as(C.POINTER(C.c_double)), st.ctypes.data_as(C.POINTER(C.c_int)),
                 ms.ctypes.data_as(C.POINTER(C.c_double)))
        ctx.close()
        assert np.all(st == 0), st
        for i in range(n):
            nk0, Nw0, dn, T, tp, tpp, t3, U = P[i]
            g = Green(int(nk0), int(Nw0), dn, T, 0.1, (tp, tpp, t3, U))
            g.set_form(_lib.FORM_NEWTON | _lib.FORM_MIXED)
            g.solve()
            ref = g.scalars()
            g.ctx.close()
            for k in ("Usp", "Uch", "mu", "dblOcc", "Sigma_inf", "trSG"):
                a, b = res[i, names.index(k)], ref[k]
                assert abs(a - b) <= 1e-11 * max(abs(b), 1e-3), (i, k, a, b)
        word = C.c_uint(0)
        assert lib.tpsc_tensor_plan_errors(C.byref(word), 1) == 0 and word.value == 0
    finally:
        for kind in range(4):
            assert lib.tpsc_set_slice_plan(kind, 256, defaults[kind]) == 0
