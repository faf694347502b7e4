"""Many points by shape groups (tpsc_solve_points): one launch per stage over
every point of a (nk0, Nw0) group, one graph launch per group, against the
one-point Newton-form mixed solve (tpsc_solve) of each point.

* Every scalar of every point agrees with its own tpsc_solve to 1e-11
  relative (the root searches' partial sums run on fewer blocks per point,
  so the last bits of the sums differ; the roots converge to 1e-14).  mu is
  measured on the root search's own scale, max(1, |mu|): its steps stop at
  1e-14 max(1, |mu|), and near half filling mu is close to 0, where a
  relative measure would ask for agreement below the search's resolution.
* A second and a third call (the captured graph, then its replay) give the
  first call's results bit for bit.
* A point with unsupported arguments gets ERR_ARG and NaN scalars; the others
  are solved.  The half-filled point without t', t'' has mu0 = 0.
* The batched sweep (tpsc_batch_* in graph mode 3) gives the per-point
  sweep's results on a sample of the sweep workload.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

def _scale(key, ref):
    """Denominator of a relative error: the root searches of mu0 and mu stop
    on steps of 1e-14 max(1, |x|), so those two take max(1, |ref|); the other
    scalars max(1e-3, |ref|)."""
    return np.maximum(np.abs(ref), 1.0 if key in ("mu0", "mu") else 1e-3)


KEYS = ("mu0", "chi0max", "Usp", "Uch", "dblOcc", "Sigma_inf", "mu", "trSG", "trSG_asymp", "trSG2", "dblOcc_SG2")


def _points():
    rows = []
    for nk0, Nw0, n, T, tp, U in [(16, 64, 0.85, 0.2, -0.1, 3.0), (16, 64, 0.95, 0.15, -0.2, 4.5),
                                  (16, 64, 1.1, 0.3, 0.0, 2.0), (32, 128, 0.875, 0.1, -0.15, 4.0),
                                  (32, 128, 1.0, 0.25, 0.0, 2.5), (12, 64, 0.9, 0.2, 0.0, 3.0),
                                  (32, 128, 0.7, 0.12, -0.3, 6.0), (64, 256, 0.9, 0.05, -0.2, 3.5)]:
        rows.append([nk0, Nw0, n, T, tp, 0.0, 0.0, U])
    return np.array(rows, dtype=np.float64)


def _solve_points(ctx, P):
    from tpsc_conductivity_b200 import _lib

    n = P.shape[0]
    res = np.zeros((n, len(_lib.SCALARS)))
    st = np.zeros(n, dtype=np.int32)
    ms = np.zeros(1)
    ctx.call("tpsc_solve_points", n, P.ctypes.data_as(C.POINTER(C.c_double)),
             res.ctypes.data_as(C.POINTER(C.c_double)), st.ctypes.data_as(C.POINTER(C.c_int)),
             ms.ctypes.data_as(C.POINTER(C.c_double)))
    return res, st


def test_groups_match_one_point_solves():
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Context, Green

    P = _points()
    ctx = Context()
    res, st = _solve_points(ctx, P)
    names = list(_lib.SCALARS)
    assert st[5] == _lib.ERR_ARG and np.all(np.isnan(res[5]))
    for i in range(P.shape[0]):
        if i == 5:
            continue
        assert st[i] == 0, (i, st[i])
        nk0, Nw0, n, T, tp, tpp, t3, U = P[i]
        g = Green(int(nk0), int(Nw0), n, T, 0.1, (tp, tpp, t3, U))
        g.set_form(_lib.FORM_NEWTON | _lib.FORM_MIXED)
        g.solve()
        ref = g.scalars()
        for k in KEYS:
            a, b = res[i, names.index(k)], ref[k]
            assert abs(a - b) <= 1e-11 * _scale(k, b), (i, k, a, b)
    assert res[4, names.index("mu0")] == 0.0
    # the graph (second call) and its replay (third) give the same numbers
    res2, st2 = _solve_points(ctx, P)
    res3, st3 = _solve_points(ctx, P)
    assert np.array_equal(st, st2) and np.array_equal(st, st3)
    ok = st == 0
    assert np.array_equal(res[ok], res2[ok]) and np.array_equal(res[ok], res3[ok])


def test_batched_sweep_mode3_matches_the_per_point_sweep():
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Batch, sweep_points

    P = sweep_points(96)
    b = Batch(4)
    ref, st_ref, _ = b.solve(P)
    b.lib.tpsc_batch_set_graph_mode(b.h, 3)
    got, st, _ = b.solve(P)
    assert np.array_equal(st, st_ref)
    names = list(_lib.SCALARS)
    for k in ("Usp", "Uch", "mu", "dblOcc", "Sigma_inf"):
        j = names.index(k)
        err = np.max(np.abs(got[:, j] - ref[:, j]) / _scale(k, ref[:, j]))
        assert err <= 1e-11, (k, err)
