"""The sum-rule tail identity the CUDA sum-rule kernel uses, checked in exact
arithmetic terms on the CPU: for chi_n = a x_n + b x_n^2 (x_n = 1/qn^2) and
h = sgn U/2,
    sum_n [chi_n/(1 + h chi_n) - chi_n] = sum_{m>=1} (-h)^m sum_i C(m+1,i) a^(m+1-i) b^i Q_(m+1+i)
with Q_k = sum_n x_n^k; truncated at m = 8 when |h chi_max| < 0.004."""
import math

import numpy as np
import pytest


def direct(a, b, h, x):
    """Term-by-term sum in the cancellation-free form -h c^2/(1 + h c) (the
    reference's c/(1+hc) - c loses ~eps/|hc| relative per term)."""
    c = a * x + b * x * x
    return float(np.sum(-h * c * c / (1 + h * c))), float(np.sum(-(c / (1 + h * c)) ** 2))


def series(a, b, h, Q, M=8):
    f = df = 0.0
    for m in range(1, M + 1):
        p = m + 1
        Sp = sum(math.comb(p, i) * a ** (p - i) * b ** i * Q[p + i] for i in range(p + 1))
        f += (-h) ** m * Sp
        df += -m * (-h) ** (m - 1) * Sp
    return f, df


@pytest.mark.parametrize("T,nw0", [(0.05, 4096), (0.25, 512), (0.1, 64)])
@pytest.mark.parametrize("a,b", [(-3.0, 40.0), (0.7, -2.0), (0.0, 5.0)])
def test_tail_series_matches_direct_sum(T, nw0, a, b):
    nwmax = nw0 // 2
    j = np.arange(nwmax + 1, 2 * nwmax + 1)
    x = 1.0 / (2 * np.pi * T * j) ** 2
    Q = [float(np.sum(x[::-1] ** k)) for k in range(20)]
    cmax = abs(a) * x[0] + abs(b) * x[0] ** 2
    for h in (0.5, -1.7, 3.0):
        if abs(h) * cmax >= 0.004:
            continue
        f, df = series(a, b, h, Q)
        fd, dfd = direct(a, b, h, x)
        assert abs(f - fd) <= 1e-13 * abs(fd) + 1e-300
        assert abs(df - dfd) <= 1e-12 * abs(dfd) + 1e-300
