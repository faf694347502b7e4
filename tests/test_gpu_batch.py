"""The batched sweep (tpsc_batch_*): many independent solves with uneven
lattices and Matsubara cutoffs on one GPU, several solver contexts at once.

Every point's scalars equal those of the same point solved alone through
tpsc_solve (tolerance 1e-11 relative: the capped cooperative root grids of a
batch sum their partials in another grouping), a failing point leaves the
others intact, and the tuner keeps one of the counts it timed."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

KEYS = ["mu0", "chi0max", "Usp", "Uch", "dblOcc", "Sigma_inf", "mu", "trSG2"]


def _single(p, form):
    from tpsc_conductivity_b200.api import Green

    g = Green(int(p[0]), int(p[1]), p[2], p[3], 0.1, (p[4], p[5], p[6], p[7]))
    g.set_form(form)
    g.solve()
    return g.scalars()


@pytest.mark.parametrize("form_name", ["newton", "mixed_newton"])
def test_batch_points_equal_single_solves(form_name):
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Batch, sweep_points

    form = _lib.FORM_NEWTON | (_lib.FORM_MIXED if form_name == "mixed_newton" else 0)
    pts = sweep_points(12, seed=7)
    b = Batch(nstreams=4)
    res, st, ms = b.solve(pts, form)
    assert np.all(st == 0) and ms > 0
    names = list(_lib.SCALARS)
    for i, p in enumerate(pts):
        ref = _single(p, form)
        for k in KEYS:
            v = res[i, names.index(k)]
            assert abs(v - ref[k]) <= 1e-11 * max(1.0, abs(ref[k])), (i, k, v, ref[k])
    # the same call again: the contexts and grids are reused, results repeat
    res2, st2, _ = b.solve(pts, form)
    assert np.all(st2 == 0)
    assert np.array_equal(res[:, [names.index(k) for k in KEYS]], res2[:, [names.index(k) for k in KEYS]])


def test_batch_reproduces_reference_scalars():
    """Golden points solved inside one batch match the reference binary."""
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Batch

    names = ["l16_w64_u2", "l32_w256_u4_tp", "l16_w128_n110", "l64_w1024_u4", "l32_w512_u2"]
    rows = []
    for nm in names:
        p = load_golden(nm)["p"]
        rows.append([p["nk0"], p["Nw0"], p["n"], p["T"], p["tp"], p["tpp"], p["t3"], p["U"]])
    b = Batch(nstreams=3)
    res, st, _ = b.solve(np.array(rows), _lib.FORM_REFERENCE)
    assert np.all(st == 0)
    sn = list(_lib.SCALARS)
    for i, nm in enumerate(names):
        s = load_golden(nm)["s"]
        for k in ("Usp", "Uch", "dblOcc", "mu"):
            assert abs(res[i, sn.index(k)] - s[k]) <= 1e-9 * max(1.0, abs(s[k])), (nm, k)


def test_batch_failing_point_is_isolated():
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Batch, sweep_points

    pts = sweep_points(6, seed=3)
    pts[2, 0] = 48  # not a supported lattice
    pts[4, 2] = 2.5  # density out of range
    b = Batch(nstreams=2)
    res, st, _ = b.solve(pts)
    assert st[2] == _lib.ERR_ARG and st[4] == _lib.ERR_ARG
    assert np.all(np.isnan(res[2])) and np.all(np.isnan(res[4]))
    ok = [i for i in range(6) if i not in (2, 4)]
    assert np.all(st[ok] == 0) and np.all(np.isfinite(res[ok, list(_lib.SCALARS).index("mu")]))


def test_batch_tuner_keeps_a_timed_count():
    from tpsc_conductivity_b200.api import Batch, sweep_points

    pts = sweep_points(16, seed=11)
    b = Batch(nstreams=1)
    t = b.tune(pts, max_streams=4)
    assert sorted(t) == [1, 2, 4] and all(v > 0 for v in t.values())
    assert b.nstreams == min(t, key=t.get)


@pytest.mark.parametrize("form_name", ["newton", "mixed_newton"])
def test_batch_as_graph_launches_equals_direct_launches(form_name):
    """Graph mode 2: every point after a grid's first runs as one launch of
    that grid's graph, updated in place for the point; the scalars are those
    of the same sweep run as direct launches, bit for bit."""
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Batch, sweep_points

    form = _lib.FORM_NEWTON | (_lib.FORM_MIXED if form_name == "mixed_newton" else 0)
    pts = sweep_points(24, seed=11)
    direct = Batch(nstreams=3)
    direct.set_graph_mode(0)
    ref, st0, _ = direct.solve(pts, form)
    graphs = Batch(nstreams=3)
    graphs.set_graph_mode(2)
    for _ in range(2):
        res, st, _ = graphs.solve(pts, form)
        assert np.array_equal(st, st0)
        ok = st0 == 0
        assert np.array_equal(res[ok], ref[ok])


def test_batch_corr_length_scan_equals_the_references_file():
    """tpsc_batch_corr_length with the reference's own semantics (the
    constructor's nsr and Fermi surface for every point) reproduces the
    reference's corrLgth file (corr_l16_w64) to 1e-8; with each point's own
    nsr, the n = 0.9 points move."""
    from tpsc_conductivity_b200.api import Batch

    g = load_golden("corr_l16_w64")
    ref = np.loadtxt(bytes(g["file_0"]).decode().splitlines(), ndmin=2)
    U, tp, tpp, t3, n, T, nk0, Nw0 = g["params"]
    nsr = n if n <= 1.0 else 2.0 - n
    b = Batch(nstreams=2)
    rows, st, ms = b.corr_length(int(nk0), int(Nw0), (tp, tpp, t3, U), g["dens"], 2, g["temp"], 2, nsr=nsr,
                                 mu_fs=ref[0, 2])
    assert not st.any() and ms > 0
    cols = [c for c in range(len(Batch.CORR_COLUMNS)) if c not in (5, 7)]
    assert np.allclose(rows[:, cols], ref[:, cols], rtol=1e-8, atol=1e-12)
    assert np.all(rows[:, [5, 7]] >= 0)
    own, st2, _ = b.corr_length(int(nk0), int(Nw0), (tp, tpp, t3, U), g["dens"], 2, g["temp"], 2)
    assert not st2.any()
    assert np.allclose(own[:2, 4], rows[:2, 4], rtol=1e-12) and np.all(np.abs(own[2:, 4] - rows[2:, 4]) > 1e-6)
