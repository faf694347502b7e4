"""The device Vidberg-Serene continued fraction (k_pade_batch) against the
oracle's recursion (generique::pade_cont_frac_coef_rec and generique::pade,
src/generique.cpp:1628-1663) on IDENTICAL inputs: the reference's own
Sigma(k, i w_n) from a fixture, every octant k, Nn = 10 (MDC,
find_FS_inter), 16 (calc_Self_Re_w_BZ) and 32 nodes.

This separates the recursion's arithmetic from its sensitivity to its
inputs.  Measured with the oracle alone, moving Sigma by two ulps moves the
continued fraction by 2e-15 (of its max) at the Matsubara nodes, by
1e-11 - 1e-9 at the next Matsubara points, and by 4e-8 (Nn = 10) to 0.7
(Nn = 16, 32) at w + 0.05i on the real axis: the continuation amplifies the
last bits of Sigma by up to 10^15.  So
  * at the nodes, where the problem is well conditioned, the device and the
    oracle agree to 1e-12 and both interpolate Sigma to 1e-12;
  * on the real axis the bound is ten times the oracle's own 2-ulp spread
    (or 1e-12, the larger): no FP64 evaluation can agree more closely, and
    the file-level tolerances of the Pade outputs (MDC, find_FS_inter,
    calc_Self_Re_w_BZ) reflect this conditioning, not the recursion.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _sigma(g):
    p = g["p"]
    S = g["self"]
    nw = S.shape[0]
    z = 1j * (2 * np.arange(nw)[:, None] + 1) * np.pi * p["T"]
    return z[:, 0], g["s"]["Sigma_inf"] / z + g["sigma_inf2"] / z ** 2 + g["sigma_inf3"] / z ** 3 + S / z ** 4


@pytest.mark.parametrize("Nn", [10, 16, 32])
def test_device_pade_recursion_matches_the_oracle_on_identical_inputs(Nn):
    from oracle import tpsc_oracle as O
    from tpsc_conductivity_b200.api import pade_batch

    g = load_golden("l32_w512_u2")
    iw, sig = _sigma(g)
    x = iw[:Nn]
    y = np.ascontiguousarray(sig[:Nn].T)             # [n8, Nn]
    zr = np.linspace(-8.0, 8.0, 200) + 0.05j
    at_nodes = pade_batch(x, y, x)
    on_axis = pade_batch(x, y, zr)
    rng = np.random.default_rng(7)
    worst_nodes, worst_axis, worst_spread = 0.0, 0.0, 0.0
    for f in range(y.shape[0]):
        coef = O.pade_coefficients(y[f], x)
        ref_n = O.pade_eval(x, x, coef)
        sn = float(np.max(np.abs(ref_n)))
        en = float(np.max(np.abs(at_nodes[f] - ref_n)))
        assert en <= 1e-12 * sn, (f, en / sn)
        assert np.max(np.abs(at_nodes[f] - y[f])) <= 1e-12 * sn
        ref = O.pade_eval(zr, x, coef)
        spread = 0.0
        for _ in range(3):
            yp = y[f] * (1.0 + 2.0 * np.finfo(float).eps * rng.choice([-1.0, 1.0], size=Nn))
            spread = max(spread, float(np.max(np.abs(O.pade_eval(zr, x, O.pade_coefficients(yp, x)) - ref))))
        scale = float(np.max(np.abs(ref)))
        err = float(np.max(np.abs(on_axis[f] - ref)))
        assert err <= max(1e-12 * scale, 10.0 * spread), (f, err / scale, spread / scale)
        worst_nodes = max(worst_nodes, en / sn)
        worst_axis = max(worst_axis, err / scale)
        worst_spread = max(worst_spread, spread / scale)
    print(f"Nn={Nn}: nodes {worst_nodes:.2e}; real axis {worst_axis:.2e} against a 2-ulp input spread "
          f"of {worst_spread:.2e}")
