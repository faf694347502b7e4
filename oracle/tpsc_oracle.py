"""CPU oracle for the TPSC hot path -- TEST INFRASTRUCTURE ONLY.

This module is a plain numpy/scipy restatement of the reference algorithm
(dbergeron1/TPSC_conductivity, C++), written from reading its sources.  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may
import it, and only as the checker: the product (``tpsc_conductivity_b200``)
never calls into it and fails loudly when its CUDA library is missing.

Parity is pinned: ``tests/test_oracle_golden.py`` checks every function here
against golden vectors produced by the unmodified reference sources compiled
in this repository (``oracle/ref/Makefile`` -> ``oracle/_ref/tpsc_ref_probe``;
fixtures and the script that made them live in ``tests/golden/``).

Conventions follow the reference:
  * lattice side ``nk0`` (L), quadrant side ``nbk = L/2+1``, octant index
    ``m + l(l+1)/2`` with ``m <= l`` (src/chi0.cpp:341);
  * ``Nw0`` = total fermionic frequency count, ``nw = Nw0/2+1`` bosonic
    n >= 0 frequencies == tau nodes on [0, beta/2];
  * 2D DCT-I == FFTW ``REDFT00`` on the nbk x nbk quadrant (unnormalised);
  * FFT of the spline third derivative uses FFTW_BACKWARD, exp(+2 pi i jk/N).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft
import scipy.linalg as sla

EPS = np.finfo(np.float64).eps
PI = math.acos(-1.0)


# ----------------------------------------------------------------------------
# lattice tables (src/hamiltonien.cpp)
# ----------------------------------------------------------------------------
def dispersion(nbk: int, tp: float, tpp: float, t3: float) -> np.ndarray:
    """eps_k on the quadrant grid k = l pi/(nbk-1); ``ek[l, m]`` with l the kx
    index (src/hamiltonien.cpp:358-375, dispk at :428-431)."""
    k = np.arange(nbk) * PI / (nbk - 1)
    kx = k[:, None]
    ky = k[None, :]
    return (-2.0 * (np.cos(kx) + np.cos(ky)) - 4.0 * tp * np.cos(kx) * np.cos(ky)
            - 2.0 * tpp * (np.cos(2 * kx) + np.cos(2 * ky))
            - 4 * t3 * (np.cos(2 * kx) * np.cos(ky) + np.cos(2 * ky) * np.cos(kx)))


def octant_index(nbk: int):
    """(l, m) arrays of the octant m <= l in storage order m + l(l+1)/2."""
    ls, ms = [], []
    for l in range(nbk):
        for m in range(l + 1):
            ls.append(l)
            ms.append(m)
    return np.array(ls), np.array(ms)


def hopping_octant(nbk: int, tp: float, tpp: float, t3: float) -> np.ndarray:
    """er[] = -t at octant sites (1,0),(1,1),(2,0),(2,1) (src/hamiltonien.cpp:17-30)."""
    n8 = nbk * (nbk + 1) // 2
    er = np.zeros(n8)
    er[1] = -1.0
    er[2] = -tp
    er[3] = -tpp
    er[4] = -t3
    return er


def octant_weights(nbk: int, base: int) -> np.ndarray:
    """Multiplicity weights of octant points: ``base`` halved on the l or m
    edges and on the diagonal (e.g. src/green0.cpp:193-196, src/chi.cpp:755-759)."""
    l, m = octant_index(nbk)
    w = np.full(l.shape, base, dtype=np.int64)
    w = np.where((l == 0) | (l == nbk - 1), w // 2, w)
    w = np.where((m == 0) | (m == nbk - 1), w // 2, w)
    w = np.where(m == l, w // 2, w)
    return w.astype(np.float64)


def to_octant(full: np.ndarray) -> np.ndarray:
    l, m = octant_index(full.shape[-1])
    return full[..., l, m]


def from_octant(oct_vals: np.ndarray, nbk: int) -> np.ndarray:
    """Symmetric nbk x nbk array from octant values (the chir_tmp fill pattern
    of src/chi0.cpp:349-358)."""
    l, m = octant_index(nbk)
    full = np.zeros(oct_vals.shape[:-1] + (nbk, nbk))
    full[..., l, m] = oct_vals
    full[..., m, l] = oct_vals
    return full


def dct2(full: np.ndarray) -> np.ndarray:
    """2D DCT-I over the last two axes, FFTW REDFT00 x REDFT00 (unnormalised)."""
    return sfft.dct(sfft.dct(full, type=1, axis=-1), type=1, axis=-2)


# ----------------------------------------------------------------------------
# root finder (src/generique.cpp:604-913 and the bounded variant :917-1234)
# ----------------------------------------------------------------------------
class RootNotFound(RuntimeError):
    pass


def _cdiv(a, b):
    """IEEE division as C does it (x/0 -> +-inf or nan, no exception)."""
    with np.errstate(all="ignore"):
        return float(np.float64(a) / np.float64(b))


def find_zero(func, init, lims=None):
    """Bracketing inverse-quadratic / secant / bisection root search with the
    reference's control flow: tol 1e-16 and 20 iterations
    (src/generique.cpp:604-913); with ``lims`` the bounded variant, tol 1e-15,
    12 iterations and eps = 2 machine epsilons (src/generique.cpp:917-1234).
    Returns (root, number_of_evaluations)."""
    if lims is None:
        tol, tol2, eps, itmax = 1.0e-16, 1.0e-10, 10.0 * EPS, 20
    else:
        tol, tol2, eps, itmax = 1.0e-15, 1.0e-10, 2.0 * EPS, 12
    nev = [0]

    def f(x):
        nev[0] += 1
        return func(x)

    nbiter = 0
    dytol = 0.01
    x0, xmin, xmax = init
    ymin = f(xmin)
    ymax = f(xmax)
    x = [x0, xmin, xmax]
    y = [0.0, ymin, ymax]
    if abs(ymin) < tol:
        return xmin, nev[0]
    if abs(ymax) < tol:
        return xmax, nev[0]
    if ymin * ymax > 0:
        y[0] = f(x[0])
        if abs(y[0]) < tol:
            return x[0], nev[0]
        if y[0] * y[2] < 0:
            xtmp = x[0]
            x[0] = (x[0] + x[2]) / 2
            x[1] = xtmp
            y[1] = y[0]
        else:
            ytmp = y[0]
            xtmp = x[0]
            if abs(y[1]) < abs(ytmp):
                ytmp, xtmp = y[1], x[1]
            if abs(y[2]) < abs(ytmp):
                ytmp, xtmp = y[2], x[2]
            xtmp1 = xtmp + 10 * eps
            ytmp1 = f(xtmp1)
            xtmp1 = xtmp - ytmp * _cdiv(xtmp1 - xtmp, ytmp1 - ytmp)
            ytmp1 = f(xtmp1)
            nbiter += 1
            while abs(ytmp1) > tol and nbiter < itmax and ytmp1 * ytmp > 0 and math.isfinite(xtmp1):
                xtmp, ytmp = xtmp1, ytmp1
                xtmp1 = xtmp + 10 * eps
                ytmp1 = f(xtmp1)
                xtmp1 = xtmp - ytmp * _cdiv(xtmp1 - xtmp, ytmp1 - ytmp)
                ytmp1 = f(xtmp1)
                nbiter += 1
            if abs(ytmp1) < tol:
                return xtmp1, nev[0]
            if ytmp1 * ytmp < 0:
                x[0] = (xtmp + xtmp1) / 2
                x[1], y[1] = xtmp, ytmp
                x[2], y[2] = xtmp1, ytmp1
            if nbiter >= itmax:
                raise RootNotFound("iteration limit in the secant search")
            if not math.isfinite(xtmp1):
                raise RootNotFound("non-finite iterate")
    if lims is not None:
        if x[1] < lims[0] or x[1] > lims[1] or x[2] < lims[0] or x[2] > lims[1]:
            raise RootNotFound("no root inside the limits")
    if abs(xmax - xmin) < eps:
        return xmin, nev[0]
    y[0] = f(x[0])
    if abs(y[0]) < tol:
        return x[0], nev[0]

    def classify():
        if y[0] * y[1] > 0:
            i1, i2 = 0, 1
        elif y[0] * y[2] > 0:
            i1, i2 = 0, 2
        else:
            i1, i2 = 1, 2
        i3 = 3 - i1 - i2
        if x[i3] > x[i1]:
            if x[i1] > x[i2]:
                far, mid = i2, i1
            else:
                far, mid = i1, i2
            im, ip = mid, i3
        else:
            if x[i1] < x[i2]:
                far, mid = i2, i1
            else:
                far, mid = i1, i2
            im, ip = i3, mid
        return i3, far, mid, im, ip

    i3, far, mid, _, _ = classify()
    x[far] = -y[mid] * _cdiv(x[i3] - x[mid], y[i3] - y[mid]) + x[mid]
    y[far] = f(x[far])
    dy = y[far]
    a = b = c = 0.0
    while abs(dy) > tol and nbiter < itmax:
        i3, far, mid, im, ip = classify()
        denom = (-x[0] * x[0] * x[2] + x[0] * x[0] * x[1] - x[0] * x[1] * x[1]
                 + x[0] * x[2] * x[2] - x[2] * x[2] * x[1] + x[2] * x[1] * x[1])
        if abs(denom) > 0.0:
            a = (x[0] * y[2] - x[0] * y[1] + x[2] * y[1] - y[2] * x[1] - y[0] * x[2] + y[0] * x[1]) / denom
            b = -(-y[2] * x[1] * x[1] + x[1] * x[1] * y[0] - x[2] * x[2] * y[0] - y[1] * x[0] * x[0]
                  + y[2] * x[0] * x[0] + y[1] * x[2] * x[2]) / denom
            c = (y[2] * x[0] * x[0] * x[1] - y[1] * x[0] * x[0] * x[2] - x[1] * x[1] * x[0] * y[2]
                 + x[2] * x[2] * x[0] * y[1] + x[1] * x[1] * y[0] * x[2] - x[2] * x[2] * y[0] * x[1]) / denom
        if (b * b - 4.0 * a * c) > 0.0 and abs(denom) > 0.0:
            sq = math.sqrt(b * b - 4.0 * a * c)
            xp = _cdiv(-b + sq, 2 * a)
            xm = _cdiv(-b - sq, 2 * a)
            if x[im] < xp < x[ip]:
                x[far] = xp
            elif x[im] < xm < x[ip]:
                x[far] = xm
            elif abs(y[i3] - y[mid]) > tol:
                x[far] = -y[mid] * (x[i3] - x[mid]) / (y[i3] - y[mid]) + x[mid]
            else:
                return x[mid], nev[0]
        else:
            if abs(y[i3] - y[mid]) > tol:
                x[far] = -y[mid] * (x[i3] - x[mid]) / (y[i3] - y[mid]) + x[mid]
            else:
                return x[mid], nev[0]
        y[far] = f(x[far])
        dyprec = abs(dy)
        dy = y[far]
        if abs(dyprec - abs(dy)) < dytol * dyprec or dyprec < abs(dy):
            x[far] = (x[i3] + x[mid]) / 2.0
            y[far] = f(x[far])
            dy = y[far]
        nbiter += 1
    best = 0
    root = x[0]
    if abs(y[1]) < abs(y[best]):
        root = x[1]
        best = 1
    if abs(y[2]) < abs(y[best]):
        root = x[2]
    return root, nev[0]


# ----------------------------------------------------------------------------
# clamped cubic spline on a uniform grid (src/generique.cpp:214-322)
# ----------------------------------------------------------------------------
def clamped_spline(V: np.ndarray, h: float, d0, dN):
    """Clamped cubic spline through V[0..N] (axis 0; extra axes are independent
    columns) with end slopes d0, dN.  Returns (a, b, c, d) per interval with
    S_j(x) = a (x-x_j)^3 + b (x-x_j)^2 + c (x-x_j) + d, the layout of
    generique::spline_coeffs_rel (src/generique.cpp:214-322).  The reference
    solves the 3N-1 banded system for (a,b,c) with LAPACK dgbsv; this restates
    the same interpolant through the node second derivatives M_j (tridiagonal
    1-4-1 system with clamped end rows), which is algebraically identical."""
    V = np.asarray(V, dtype=np.float64)
    N = V.shape[0] - 1
    rhs = np.empty_like(V)
    rhs[1:N] = 6.0 / (h * h) * (V[2:] - 2.0 * V[1:N] + V[:N - 1])
    rhs[0] = 6.0 / h * ((V[1] - V[0]) / h - d0)
    rhs[N] = 6.0 / h * (dN - (V[N] - V[N - 1]) / h)
    ab = np.zeros((3, N + 1))
    ab[0, 1:] = 1.0
    ab[1, :] = 4.0
    ab[1, 0] = 2.0
    ab[1, N] = 2.0
    ab[2, :-1] = 1.0
    M = sla.solve_banded((1, 1), ab, rhs.reshape(N + 1, -1)).reshape(V.shape)
    a = (M[1:] - M[:-1]) / (6.0 * h)
    b = M[:-1] / 2.0
    c = (V[1:] - V[:-1]) / h - h * (2.0 * M[:-1] + M[1:]) / 6.0
    d = V[:-1]
    return a, b, c, d


# ----------------------------------------------------------------------------
# green0: mu0 on the finite lattice (src/green0.cpp:182-203, 240-262)
# ----------------------------------------------------------------------------
def mu0_finite(ek: np.ndarray, n: float, T: float, tp=0.0, tpp=0.0):
    if n == 1.0 and tp == 0 and tpp == 0:
        return 0.0
    nbk = ek.shape[0]
    w = octant_weights(nbk, 8)
    eo = to_octant(ek)
    nk2 = 4 * (nbk - 1) * (nbk - 1)

    def dens(mup):
        return float(np.sum(2 * w / ((np.exp((eo - mup) / T) + 1.0) * nk2))) - n

    root, _ = find_zero(dens, (0.0, -8.0, 8.0))
    return root


# ----------------------------------------------------------------------------
# chi0 (src/chi0.cpp:279-718)
# ----------------------------------------------------------------------------
@dataclass
class Chi0Result:
    chiqw: np.ndarray          # [nw, N8]  chi0(q, iqn), n = 0..Nw0/2
    chirt: np.ndarray          # [nw, N8]  chi0(r, tau_j)
    chi0_inf: np.ndarray       # [N8]      coefficient of 1/qn^2
    chi0_inf2: np.ndarray      # [N8]      coefficient of 1/qn^4
    dtau_chirt0: np.ndarray    # [N8]      d/dtau chi0(r, 0)
    dtau_Grt0p: np.ndarray     # [N8]      d/dtau G(r, 0+)
    dtau_chiqt0: np.ndarray    # [N8]      d/dtau chi0(q, 0)
    chi0max: float
    qmax: tuple


def chi0_fft_spline(ek: np.ndarray, mu0: float, T: float, er: np.ndarray, nw0: int) -> Chi0Result:
    """chi0::calc_chiqw_FFT_spline (src/chi0.cpp:279-718)."""
    nk = ek.shape[0]
    nq0 = 2 * (nk - 1)
    nk02 = float(nq0 * nq0)
    nw = nw0 // 2 + 1
    n8 = nk * (nk + 1) // 2
    beta = 1.0 / T
    ekmu = to_octant(ek) - mu0                                   # :341
    Gkt = -1.0 / (np.exp(-ekmu / T) + 1.0)                       # :342

    # d/dtau G(r, 0-) and d/dtau G(r, 0+) (:323-367)
    dG0m = er.copy()
    dG0m[0] = -mu0
    tmp = to_octant(dct2(from_octant(-ekmu * Gkt / nk02, nk)))
    dG0m = dG0m - tmp
    dG0p = tmp

    # G(r, 0+) and chi0(r, 0) (:375-418)
    G0 = to_octant(dct2(from_octant(Gkt / nk02, nk)))
    chir = -2.0 * G0 * G0
    chir[0] = -2.0 * G0[0] * (G0[0] + 1.0)
    chirt = np.empty((nw, n8))
    chiqt = np.empty((nw, n8))
    chirt[0] = chir
    chiqt[0] = to_octant(dct2(from_octant(chir, nk)))

    # d/dtau chi0(r, 0) (:424-447)
    dchir = -2.0 * (dG0p * G0 + dG0m * G0)
    dchir[0] = -2.0 * (dG0p[0] * (1.0 + G0[0]) + dG0m[0] * G0[0])
    dtau_chiqt0 = to_octant(dct2(from_octant(dchir, nk)))

    # 0 < tau < beta/2 (:454-519)
    pos = ekmu >= 0.0
    ex = np.exp(ekmu / T)
    for j in range(1, nw - 1):
        t = j / (nw0 * T)
        gp = np.where(pos, np.exp(-t * ekmu) * Gkt / nk02,
                      -np.exp((beta - t) * ekmu) / (ex + 1.0) / nk02)
        gm = np.where(pos, -np.exp((t - beta) * ekmu) * Gkt / nk02,
                      np.exp(t * ekmu) / ((ex + 1.0) * nk02))
        Gp = to_octant(dct2(from_octant(gp, nk)))
        Gm = to_octant(dct2(from_octant(gm, nk)))
        chir = -2.0 * Gm * Gp
        chirt[j] = chir
        chiqt[j] = to_octant(dct2(from_octant(chir, nk)))
    # tau = beta/2 (:527-559)
    j = nw - 1
    t = 1.0 / (2.0 * T)
    gp = np.where(pos, np.exp(-t * ekmu) * Gkt / nk02,
                  -np.exp((beta - t) * ekmu) / ((ex + 1.0) * nk02))
    Gp = to_octant(dct2(from_octant(gp, nk)))
    chir = 2.0 * Gp * Gp
    chirt[j] = chir
    chiqt[j] = to_octant(dct2(from_octant(chir, nk)))

    # per q: clamped spline along tau, FFT of 6 a_j, tails (:586-690)
    h = 1.0 / (nw0 * T)
    a, b, c, d = clamped_spline(chiqt, h, dtau_chiqt0, np.zeros(n8))
    f = np.empty((nw0, n8))
    f[: nw0 // 2] = 6.0 * a
    f[nw0 // 2:] = -f[: nw0 // 2][::-1]
    F = np.fft.ifft(f, axis=0) * nw0                            # FFTW_BACKWARD
    x = h
    integ = np.sum(a * x ** 4 / 4.0 + b * x ** 3 / 3.0 + c * x ** 2 / 2.0 + d * x, axis=0)
    chiqw = np.empty((nw, n8))
    chiqw[0] = 2 * integ
    chi0_inf = -2.0 * dtau_chiqt0
    jj = np.arange(1, nw)[:, None]
    wn = 2 * jj * PI * T
    th = 2 * jj * PI / nw0
    chiqw[1:] = chi0_inf / (wn * wn) + ((1.0 - np.cos(th)) * F[1:nw].real
                                        + np.sin(th) * F[1:nw].imag) / (wn ** 4)
    chi0_inf2 = 2.0 * F[nw - 1].real
    chi0_inf[0] = 0.0
    chi0_inf2[0] = 0.0
    chiqw[1:, 0] = 0.0

    # chi0max and its wave vector (:703-717): scan l down, m down, strict >
    chi0max = 0.0
    qmax = (0, 0)
    for l in range(nk - 1, -1, -1):
        for m in range(l, -1, -1):
            v = chiqw[0, m + l * (l + 1) // 2]
            if v > chi0max:
                chi0max = v
                qmax = (l, m)
    return Chi0Result(chiqw, chirt, chi0_inf, chi0_inf2, dchir, dG0p, dtau_chiqt0, chi0max, qmax)


def trace_chi0(r: Chi0Result, n: float, T: float):
    """chi0::traceChi0 (src/chi0.cpp:1498-1584) -> (raw trace, extrapolated)."""
    nw, n8 = r.chiqw.shape
    nk = int(round((math.sqrt(8 * n8 + 1) - 1) / 2))
    nwmax = nw - 1
    Nq = 4 * (nk - 1) ** 2
    w = octant_weights(nk, 16)
    wj = np.ones(nw)
    wj[0] = 0.5
    wj[nwmax] = 0.5
    tr1 = float(np.sum(wj[:, None] * w[None, :] * T * r.chiqw / Nq))
    jj = np.arange(nwmax + 1, 2 * nwmax)[:, None]
    wn = 2 * PI * jj * T
    c = r.chi0_inf / (wn * wn) + r.chi0_inf2 / wn ** 4
    tr = tr1 + float(np.sum(w * T * c / Nq))
    N1 = nwmax + 1
    tr_corr = tr + N1 * (tr1 - tr) / (N1 - 2 * nwmax)
    return tr, tr_corr


# ----------------------------------------------------------------------------
# chi: sum rules and Usp, Uch (src/chi.cpp:738-876, 210-371)
# ----------------------------------------------------------------------------
def trace_diff_chi(r: Chi0Result, Uv: float, sign: float, T: float) -> float:
    """traceDiffChispChi0 (sign=-1) / traceDiffChichChi0 (sign=+1)
    (src/chi.cpp:738-830): sum of chi0/(1 + sign*U chi0/2) - chi0, stored
    frequencies n <= Nw0/2 plus tails Nw0/2 < n <= Nw0."""
    nw, n8 = r.chiqw.shape
    nk = int(round((math.sqrt(8 * n8 + 1) - 1) / 2))
    nwmax = nw - 1
    Nq = 4 * (nk - 1) ** 2
    w = octant_weights(nk, 16)
    jj = np.arange(nwmax + 1, 2 * nwmax + 1)[:, None]
    wn = 2 * jj * PI * T
    c = r.chi0_inf / (wn * wn) + r.chi0_inf2 / (wn * wn * wn * wn)
    tail = np.sum(w * T / Nq * (c / (1 + sign * Uv * c / 2.0) - c))
    wj = np.ones(nw)
    wj[0] = 0.5
    c = r.chiqw
    main = np.sum(wj[:, None] * w[None, :] * T / Nq * (c / (1 + sign * Uv * c / 2.0) - c))
    return float(main + tail)


@dataclass
class UResult:
    Usp: float
    Uch: float
    dblOcc: float
    evals_sp: int
    evals_ch: int


def find_Usp_Uch(r: Chi0Result, U: float, n: float, T: float) -> UResult:
    """chi::find_Usp_Uch(nq0, nw0, Usc) on one grid (src/chi.cpp:846-876) and
    the double occupancy ansatz (src/chi.cpp:370-371)."""
    nsr = 2.0 - n if n > 1.0 else n

    def rsp(Us):
        return trace_diff_chi(r, Us, -1.0, T) + n - n * n / 2.0 - nsr + Us * nsr * nsr / (2.0 * U)

    Usp, ev1 = find_zero(rsp, (U / 2.0, 0.0, 2.0 / r.chi0max - 2 * EPS))

    def rch(Uc):
        return trace_diff_chi(r, Uc, 1.0, T) + n - n * n / 2.0 - (nsr + Usp * nsr * nsr / (2.0 * U) - nsr * nsr)

    Uch, ev2 = find_zero(rch, (0.0, 0.0, 1000.0 * U))
    if n > 1.0:
        D = Usp / U * nsr * nsr / 4.0 + 1.0 - nsr
    else:
        D = Usp / U * nsr * nsr / 4.0
    return UResult(Usp, Uch, D, ev1, ev2)


def vertex_rt(r: Chi0Result, U: float, Usp: float, Uch: float, T: float) -> np.ndarray:
    """chi::calc_chirt (src/chi.cpp:37-170): V(r, tau_j), j = 0..Nw0/2."""
    nw, n8 = r.chiqw.shape
    nk = int(round((math.sqrt(8 * n8 + 1) - 1) / 2))
    nq0 = 2 * (nk - 1)
    normFact = T / (nq0 * nq0)
    c0 = r.chiqw
    csp = c0 / (1.0 - Usp * c0 / 2.0)
    cch = c0 / (1.0 + Uch * c0 / 2.0)
    vq = normFact * U * (3.0 * Usp * (csp - c0) + Uch * (cch - c0)) / 8.0
    vr = to_octant(dct2(from_octant(vq, nk)))
    vr = sfft.dct(vr, type=1, axis=0)
    return vr + U * (3.0 * Usp + Uch) / 8.0 * r.chirt


# ----------------------------------------------------------------------------
# green: self-energy (src/green.cpp:1673-2025)
# ----------------------------------------------------------------------------
@dataclass
class SelfResult:
    S: np.ndarray            # [Nw0/2, N8] complex: coefficient of 1/z^4
    Sigma_inf: float         # coefficient of 1/z (k-independent)
    Sigma_inf2: np.ndarray   # [N8] coefficient of 1/z^2
    Sigma_inf3: np.ndarray   # [N8] coefficient of 1/z^3
    Sigma_inf4: np.ndarray   # [N8] Re S at the last stored frequency
    sigma_tau: np.ndarray = field(repr=False, default=None)   # [Nw0+1, N8]

    def sigma(self, T: float) -> np.ndarray:
        """Full Sigma(k, i w_n) for n < Nw0/2 (src/green.cpp:3039)."""
        nj = self.S.shape[0]
        z = 1j * (2 * np.arange(nj)[:, None] + 1) * PI * T
        return (self.Sigma_inf / z + self.Sigma_inf2 / (z * z) + self.Sigma_inf3 / (z * z * z)
                + self.S / (z * z * z * z))


def self_energy(ek, mu0, T, er, r: Chi0Result, V: np.ndarray, U, Usp, Uch, nbw) -> SelfResult:
    """green::calc_Self_FFT_spline, stages after calc_chirt (src/green.cpp:1741-2025)."""
    nk = ek.shape[0]
    nk0 = 2 * (nk - 1)
    nk02 = float(nk0 * nk0)
    n8 = nk * (nk + 1) // 2
    nw = nbw // 2 + 1
    ekmu = ek - mu0
    fact = U * (3.0 * Usp + Uch) / 8.0

    # d/dtau Sigma(k, 0) and d/dtau Sigma(k, beta) (:1745-1817)
    g = to_octant(dct2(-1.0 / (np.exp(-ekmu / T) + 1.0) / nk02))
    s0 = (fact * r.dtau_chirt0) * g + V[0] * r.dtau_Grt0p
    d0 = to_octant(dct2(from_octant(s0, nk)))
    g = to_octant(dct2(-1.0 / (np.exp(ekmu / T) + 1.0) / nk02))
    xi = er.copy()
    xi[0] = -mu0
    sb = (-fact * r.dtau_chirt0) * g + V[0] * (-r.dtau_Grt0p + xi)
    dN = to_octant(dct2(from_octant(sb, nk)))

    # Sigma(k, tau_j), j = 0..Nw0 (:1822-1885)
    st = np.empty((nbw + 1, n8))
    pos = ekmu > 0
    e1 = np.exp(-ekmu / T) + 1.0
    e2 = np.exp(ekmu / T) + 1.0
    for j in range(nbw + 1):
        t = j / (nbw * T)
        gk = np.where(pos, -np.exp(-t * ekmu) / e1 / nk02, -np.exp((1.0 / T - t) * ekmu) / e2 / nk02)
        gr = to_octant(dct2(gk))
        vr = V[j] if j < nw else V[nbw - j]
        st[j] = to_octant(dct2(from_octant(gr * vr, nk)))

    # per k: spline over [0, beta], FFT, tails (:1935-2017)
    h = 1.0 / (nbw * T)
    a, b, c, d = clamped_spline(st, h, d0, dN)
    d2S0 = 2 * b[0]
    d2Sb = 6.0 * a[nbw - 1] / (nbw * T) + 2.0 * b[nbw - 1]
    jj = np.arange(nbw)[:, None]
    f = np.exp(1j * jj * PI / nbw) * 6.0 * a
    F = np.fft.ifft(f, axis=0) * nbw
    coeff1 = st[0] + st[nbw]
    Sigma_inf = float(-coeff1[0])
    S2 = d0 + dN
    S3 = -(d2S0 + d2Sb)
    jh = np.arange(nbw // 2)[:, None]
    S = (1.0 - np.exp(1j * (2 * jh + 1) * PI / nbw)) * F[: nbw // 2]
    S4 = S[nbw // 2 - 1].real.copy()
    return SelfResult(S, Sigma_inf, S2, S3, S4, st)


def _sigma_parts(sr: SelfResult, T: float):
    sig = sr.sigma(T)
    return sig.real, sig.imag


def trace_self_G(ek, mu0, sr: SelfResult, T: float):
    """green::traceSelfG (src/green.cpp:3001-3089) -> (sum, sum + asymptotic)."""
    nk = ek.shape[0]
    nk02 = 4 * (nk - 1) ** 2
    w = octant_weights(nk, 8)
    eo = to_octant(ek)
    nj = sr.S.shape[0]
    wn = (2 * np.arange(nj)[:, None] + 1) * PI * T
    rS, iS = _sigma_parts(sr, T)
    tmp = w * T * 2 / (nk02 * (wn * wn + (eo - mu0) ** 2))
    s = float(np.sum(tmp * (rS * (mu0 - eo) + iS * wn)))
    s2 = float(np.sum(w * sr.Sigma_inf * T * 2 / (nk02 * (wn * wn + (eo - mu0) ** 2))))
    x = eo - mu0
    big = np.abs(x) > 1.0e-12
    ek_ = np.where(x < 0, np.exp(x / T), np.exp(-x / T))
    s2 += float(np.sum(np.where(big, w * sr.Sigma_inf * (1.0 / (np.exp(x / T) + 1.0) - 0.5) / np.where(big, x, 1.0) / nk02,
                                -w * sr.Sigma_inf * ek_ / ((ek_ + 1.0) * (ek_ + 1.0) * nk02 * T))))
    return s, s + s2


def trace_diff_G(ek, mu0, sr: SelfResult, T: float, pmu: float) -> float:
    """green::traceDiffG (src/green.cpp:3108-3182): Tr(G - G0) at chemical
    potential pmu, stored frequencies plus the analytic tail up to j = Nw0."""
    nk = ek.shape[0]
    w = octant_weights(nk, 16)
    eo = to_octant(ek)
    nj = sr.S.shape[0]
    nbw = 2 * nj
    jt = np.arange(nbw // 2, nbw + 1)[:, None]
    wn = (2 * jt + 1) * PI * T
    rS = -sr.Sigma_inf2 / (wn * wn) + sr.Sigma_inf4 / (wn * wn * wn * wn)
    iS = -sr.Sigma_inf / wn + sr.Sigma_inf3 / (wn * wn * wn)
    tmp = w / (((wn - iS) ** 2 + (eo - pmu + rS) ** 2) * (wn * wn + (eo - mu0) ** 2))
    s1 = np.sum(tmp * ((mu0 - pmu + rS) * (eo - pmu + rS) * (eo - mu0) + iS * (iS - 2 * wn) * (eo - mu0)
                       - wn * wn * (mu0 - pmu + rS)))
    wn = (2 * np.arange(nj)[:, None] + 1) * PI * T
    rS, iS = _sigma_parts(sr, T)
    tmp = w / (((wn - iS) ** 2 + (eo - pmu + rS) ** 2) * (wn * wn + (eo - mu0) ** 2))
    s = np.sum(tmp * ((mu0 - pmu + rS) * (eo - pmu + rS) * (eo - mu0) + iS * (iS - 2 * wn) * (eo - mu0)
                      - wn * wn * (mu0 - pmu + rS)))
    return float(s + s1)


def find_mu(ek, mu0, sr: SelfResult, T: float):
    """green::find_mu (src/green.cpp:3185-3259)."""
    return find_zero(lambda m: trace_diff_G(ek, mu0, sr, T, m), (0.0, -10.0, 10.0), lims=(-20.0, 20.0))


def trace_self_G2(ek, mu, sr: SelfResult, T: float, U: float, n: float):
    """green::traceSelfG2 (src/green.cpp:2929-2980) -> (trace, double occupancy)."""
    nk = ek.shape[0]
    nk02 = 4 * (nk - 1) ** 2
    w = octant_weights(nk, 8)
    eo = to_octant(ek)
    nj = sr.S.shape[0]
    wn = (2 * np.arange(nj)[:, None] + 1) * PI * T
    rS, iS = _sigma_parts(sr, T)
    tmp = w * T * 2 / (nk02 * ((wn - iS) ** 2 + (eo - mu + rS) ** 2))
    s = float(np.sum(tmp * (iS * wn - iS * iS - (eo - mu) * rS - rS * rS)))
    return s, (s + U * n * n / 4.0) / U


# ----------------------------------------------------------------------------
# one full solve in the reference's order (src/tpsc_main.cpp:61-75)
# ----------------------------------------------------------------------------
@dataclass
class Solve:
    nk0: int
    Nw0: int
    mu0: float
    chi0: Chi0Result
    U: UResult
    V: np.ndarray
    sigma: SelfResult
    mu: float
    trace_self_G: tuple
    trace_self_G2: tuple


def solve(U, tp, tpp, t3, n, T, nk0, Nw0) -> Solve:
    """Full-grid TPSC solve: chi0 -> Usp, Uch -> V(r,tau) -> Sigma -> mu.  The
    reference's half-grid Usp/Uch pre-pass (src/chi.cpp:285-297) only feeds the
    difRel diagnostics, so it is not part of the solve."""
    nbk = nk0 // 2 + 1
    ek = dispersion(nbk, tp, tpp, t3)
    er = hopping_octant(nbk, tp, tpp, t3)
    mu0 = mu0_finite(ek, n, T, tp, tpp)
    c0 = chi0_fft_spline(ek, mu0, T, er, Nw0)
    ur = find_Usp_Uch(c0, U, n, T)
    V = vertex_rt(c0, U, ur.Usp, ur.Uch, T)
    sr = self_energy(ek, mu0, T, er, c0, V, U, ur.Usp, ur.Uch, Nw0)
    tsg = trace_self_G(ek, mu0, sr, T)
    mu, _ = find_mu(ek, mu0, sr, T)
    tsg2 = trace_self_G2(ek, mu, sr, T, U, n)
    return Solve(nk0, Nw0, mu0, c0, ur, V, sr, mu, tsg, tsg2)


# ----------------------------------------------------------------------------
# real-frequency continuation and local G (src/generique.cpp:1605-1663,
# src/green.cpp:209-266, 814-1068, 2210-2341)
# ----------------------------------------------------------------------------
def pade_coefficients(f, x):
    """Vidberg-Serene continued-fraction coefficients
    (generique::pade_cont_frac_coef_rec / pade_recursion, src/generique.cpp:1649-1663):
    g_0(l) = f_l, g_m(l) = (g_{m-1}(m-1) - g_{m-1}(l)) / ((x_l - x_{m-1}) g_{m-1}(l)),
    coef_m = g_m(m)."""
    N = len(f)
    g = np.array(f, dtype=np.complex128)
    coef = np.zeros(N, dtype=np.complex128)
    coef[0] = g[0]
    for m in range(1, N):
        gm = g[m - 1]
        g[m:] = (gm - g[m:]) / ((x[m:] - x[m - 1]) * g[m:])
        coef[m] = g[m]
    return coef


def pade_eval(z, x0, coef):
    """generique::pade (src/generique.cpp:1628-1646)."""
    n = len(coef)
    A = 1.0 + 0j
    B = 1.0 + (z - x0[0]) * coef[1]
    q = A / B
    for j in range(3, n + 1):
        A = 1.0 + (z - x0[j - 2]) * coef[j - 1] / A
        B = 1.0 + (z - x0[j - 2]) * coef[j - 1] / B
        q = q * A / B
    return q * coef[0]


def lagrange_eval(z, x0, f):
    s = 0j
    for j in range(len(f)):
        t = f[j]
        for i in range(len(f)):
            if i != j:
                t = t * (z - x0[i]) / (x0[j] - x0[i])
        s += t
    return s


def pade_sigma(ek, mu, sr: SelfResult, T, z, n_idx, Nn, mode=0):
    """Sigma(k, z) and A(k, z) for every octant k from Nn Matsubara samples read at
    the stored frequency j with z_j = i (2 n_idx[j] + 1) pi T (green::MDC,
    src/green.cpp:986-1003): mode 0 Pade, mode 1 Lagrange polynomial."""
    eo = to_octant(ek)
    sig = sr.sigma(T)
    x0 = 1j * (2 * np.asarray(n_idx[:Nn]) + 1) * PI * T
    z = np.atleast_1d(np.asarray(z, dtype=np.complex128))
    out_s = np.zeros((eo.size, z.size), dtype=np.complex128)
    out_A = np.zeros((eo.size, z.size))
    for o in range(eo.size):
        f = sig[:Nn, o]
        coef = pade_coefficients(f, x0) if mode == 0 else None
        for iz, zz in enumerate(z):
            s = pade_eval(zz, x0, coef) if mode == 0 else lagrange_eval(zz, x0, f)
            out_s[o, iz] = s
            out_A[o, iz] = -(1.0 / (zz - (eo[o] - mu) - s)).imag / PI
    return out_s, out_A


def fs_inter(ek, mu, sr: SelfResult, T):
    """green::find_FS_inter (src/green.cpp:2210-2341): along each line
    (l + m, m) of the quadrant, the m maximising A(k, w = 0 + i 1e-6) from a
    3-point polynomial and from a 4-point Pade; rows (l + m*, m*, A*)."""
    nbk = ek.shape[0]
    z = 1e-6j
    _, A_poly = pade_sigma(ek, mu, sr, T, [z], np.arange(3), 3, mode=1)
    _, A_pade = pade_sigma(ek, mu, sr, T, [z], np.arange(4), 4, mode=0)
    res_poly, res_pade = [], []
    for l in range(nbk):
        for A, res in ((A_poly, res_poly), (A_pade, res_pade)):
            best, bm = 0.0, 0
            for m in range(nbk - l):
                x, y = l + m, m
                a = A[y + x * (x + 1) // 2, 0]
                if a > best:
                    best, bm = a, m
            res.append((l + bm, bm, best))
    return np.array(res_poly), np.array(res_pade)


def gwn_local(ek, mu, sr: SelfResult, T):
    """green::Gwn_local (src/green.cpp:209-266)."""
    nbk = ek.shape[0]
    nk02 = 4 * (nbk - 1) ** 2
    w = octant_weights(nbk, 8)
    eo = to_octant(ek)
    sig = sr.sigma(T)
    z = 1j * (2 * np.arange(sig.shape[0])[:, None] + 1) * PI * T
    return np.sum((w / nk02) / (z - eo + mu - sig), axis=1)


# ----------------------------------------------------------------------------
# current-current correlator: bubble + Maki-Thompson and kx0
# (cond_opt::calc_chijj_vertex_corr_all_optim with chi3 = false,
# src/cond_opt.cpp:2537-4286)
# ----------------------------------------------------------------------------
def grad_ek_x(kx, ky, tp, tpp, t3):
    """d eps/d kx (hamiltonien::grad_ek dir 0, src/hamiltonien.cpp:134-142)."""
    return (2.0 * np.sin(kx) + 4.0 * tp * np.sin(kx) * np.cos(ky) + 4.0 * tpp * np.sin(2 * kx)
            + 4 * t3 * (2.0 * np.sin(2 * kx) * np.cos(ky) + np.cos(2 * ky) * np.sin(kx)))


def hessian_ek_xx(kx, ky, tp, tpp, t3):
    """d2 eps/d kx2 (hamiltonien::Hessian_ek (0,0), src/hamiltonien.cpp:145-155)."""
    return (2.0 * np.cos(kx) + 4.0 * tp * np.cos(kx) * np.cos(ky) + 8.0 * tpp * np.cos(2 * kx)
            + 4 * t3 * (4.0 * np.cos(2 * kx) * np.cos(ky) + np.cos(2 * ky) * np.cos(kx)))


def dst_dct(a):
    """FFTW RODFT00 along axis -2 and REDFT00 along axis -1 (unnormalised)."""
    return sfft.dst(sfft.dct(a, type=1, axis=-1), type=1, axis=-2)


def find_roots_2pol(A, B, C):
    """generique::find_roots_2pol (src/generique.cpp:1666-1727): roots of
    A z^2 + B z + C, then Newton polish (tol 1e-16, <= 10 steps), elementwise."""
    R = np.sqrt(B * B - 4.0 * A * C + 0j)
    roots = [(-B - R) / (2.0 * A), (-B + R) / (2.0 * A)]
    out = []
    for r0 in roots:
        x = np.array(r0, dtype=np.complex128)
        y = A * x * x + B * x + C
        p = 2.0 * A * x + B
        y0 = y.copy()
        for _ in range(10):
            act = (np.abs(p) > 0) & (np.abs(y) > 1e-16)
            if not np.any(act):
                break
            x2, y2 = x.copy(), y.copy()
            c = y - p * x
            xn = np.where(act, -c / np.where(act, p, 1), x)
            yn = A * xn * xn + B * xn + C
            worse = act & (np.abs(y2) < np.abs(yn))
            xn = np.where(worse, 0.5 * (xn + x2), xn)
            x = xn
            y = A * x * x + B * x + C
            p = 2.0 * A * x + B
        out.append(np.where(np.abs(y) < np.abs(y0), x, r0))
    return out


@dataclass
class CondResult:
    chijj1: np.ndarray   # [Nw0/2 + 1] bubble chi_jj(iqn)
    chijj2: np.ndarray   # [Nw0/2 + 1] Maki-Thompson correction
    kx0: float           # diamagnetic term <-kx> (f-sum: chijj1(0)+chijj2(0) = -kx0)
    chijj1_k: np.ndarray = None   # [Nw0/2 + 1, ntheta] angle-resolved
    chijj2_k: np.ndarray = None


def conductivity(sv: Solve, tp, tpp, t3, U, T, ntheta=1) -> CondResult:
    nk0, nbw = sv.nk0, sv.Nw0
    nbk = nk0 // 2 + 1
    n8 = nbk * (nbk + 1) // 2
    nw = nbw // 2
    ek = dispersion(nbk, tp, tpp, t3)
    mu0, mu = sv.mu0, sv.mu
    sr, V, c0 = sv.sigma, sv.V, sv.chi0
    Usp, Uch = sv.U.Usp, sv.U.Uch
    normFact = 1.0 / (nk0 * nk0)
    kq = np.arange(nbk) * PI / (nbk - 1)
    # tables (src/cond_opt.cpp:2588-2611)
    d2ek = hessian_ek_xx(kq[:, None], kq[None, :], tp, tpp, t3)                 # [nbk, nbk]
    dek = grad_ek_x(kq[1:nbk - 1, None], kq[None, :], tp, tpp, t3)              # [nbk-2, nbk]
    xk = ek[1:nbk - 1, :] - mu0                                                # eps - mu0 on K4
    pos = xk > 0
    # h(r, tau_j) (:2696-2735)
    h = np.empty((nbw + 1, nbk - 2, nbk))
    for j in range(nbw + 1):
        t = j / (T * nbw)
        fr = np.where(pos, normFact * dek * np.exp(-xk * t) / (np.exp(-xk / T) + 1.0),
                      normFact * dek * np.exp(xk * (1.0 / T - t)) / (np.exp(xk / T) + 1.0))
        h[j] = dst_dct(fr)
    # dh at tau = 0, beta (:2744-2783)
    dh0 = dst_dct(np.where(pos, -normFact * dek * xk / (np.exp(-xk / T) + 1.0),
                           -normFact * dek * xk * np.exp(xk / T) / (np.exp(xk / T) + 1.0)))
    dhb = dst_dct(np.where(pos, -normFact * dek * xk * np.exp(-xk / T) / (np.exp(-xk / T) + 1.0),
                           -normFact * dek * xk / (np.exp(xk / T) + 1.0)))
    # f0(r, tau_j) (:2794-2827)
    f0 = np.empty_like(h)
    ekp = np.exp(-xk / T)
    ekn = np.exp(xk / T)
    for j in range(nbw + 1):
        t = j / (T * nbw)
        fr = np.where(pos,
                      normFact * dek * np.exp(-xk * t) * (t / (ekp + 1.0) - ekp / (T * (ekp + 1.0) ** 2)),
                      normFact * dek * np.exp(xk * (1.0 / T - t)) * (t / (ekn + 1.0) - 1.0 / (T * (ekn + 1.0) ** 2)))
        f0[j] = dst_dct(fr)
    # df0 at tau = 0, beta (:2835-2887)
    df00 = dst_dct(np.where(pos, normFact * dek * (xk * ekp / (T * (ekp + 1.0) ** 2) + 1.0 / (ekp + 1.0)),
                            normFact * dek * ekn * (xk / (T * (ekn + 1.0) ** 2) + 1.0 / (ekn + 1.0))))
    df0b = dst_dct(np.where(pos, normFact * dek * ekp * ((-xk) * (1.0 / (T * (ekp + 1.0)) - ekp / (T * (ekp + 1.0) ** 2))
                                                        + 1.0 / (ekp + 1.0)),
                            normFact * dek * ((-xk) * (1.0 / (T * (ekn + 1.0)) - 1.0 / (T * (ekn + 1.0) ** 2))
                                              + 1.0 / (ekn + 1.0))))
    # vertex on the K4-shaped r grid: r = (l+1, m) folded into the octant (:2892-2908)
    lx = np.arange(1, nbk - 1)[:, None] * np.ones((1, nbk), dtype=int)
    my = np.ones((nbk - 2, 1), dtype=int) * np.arange(nbk)[None, :]
    xo = np.maximum(lx, my)
    yo = np.minimum(lx, my)
    oidx = yo + xo * (xo + 1) // 2
    fact = U * (3.0 * Usp + Uch) / 4
    V0 = V[0][oidx]
    dchi = c0.dtau_chirt0[oidx]
    dhV0 = dst_dct(2.0 * dh0 * V0 + h[0] * fact * dchi)
    dhVb = dst_dct(2.0 * dhb * V0 - h[nbw] * fact * dchi)
    df0V0 = dst_dct(2.0 * df00 * V0 + f0[0] * fact * dchi)
    df0Vb = dst_dct(2.0 * df0b * V0 - f0[nbw] * fact * dchi)
    for j in range(nbw + 1):
        wn = j if j <= nbw // 2 else nbw - j
        h[j] = dst_dct(2.0 * h[j] * V[wn][oidx])
        f0[j] = dst_dct(2.0 * f0[j] * V[wn][oidx])
    # per k (:3179-3871), vectorised over the K4 grid; axis 0 = tau or frequency
    K = (nbk - 2) * nbk
    hk = h.reshape(nbw + 1, K)
    f0k = f0.reshape(nbw + 1, K)
    ok = oidx.reshape(K)
    e = ek[1:nbk - 1, :].reshape(K)
    wt = np.where((my == 0) | (my == nbk - 1), 2.0, 4.0).reshape(K)
    dk = dek.reshape(K)
    hdt = 1.0 / (nbw * T)
    jj = np.arange(nbw)[:, None]

    def spline_to_matsubara(vals, d0, dN):
        """J(i k_n) for the nbw fermionic frequencies in the reference's
        ordering (index p <-> n = p - nbw/2) (:3204-3234)."""
        a, b, c, d = clamped_spline(vals, hdt, d0, dN)
        F = np.fft.ifft(np.exp(1j * jj * PI / nbw) * 6.0 * a, axis=0) * nbw
        C1 = -vals[0] - vals[nbw]
        C2_ = d0 + dN
        d2J0 = 2 * b[0]
        d2Jb = 6.0 * a[nbw - 1] / (nbw * T) + 2.0 * b[nbw - 1]
        C3_ = -d2J0 - d2Jb
        out = np.empty((nbw, K), dtype=np.complex128)
        jpos = np.arange(nbw // 2)[:, None]
        kn = (2 * jpos + 1) * PI * T
        out[jpos[:, 0] + nbw // 2] = (-1j * C1 / kn - C2_ / kn ** 2 + 1j * C3_ / kn ** 3
                                      + (1.0 - np.exp(1j * (2 * jpos + 1) * PI / nbw)) * F[:nbw // 2] / kn ** 4)
        jneg = np.arange(nbw // 2, nbw)[:, None]
        kn = (2 * (jneg - nbw) + 1) * PI * T
        out[jneg[:, 0] - nbw // 2] = (-1j * C1 / kn - C2_ / kn ** 2 + 1j * C3_ / kn ** 3
                                      + (1.0 - np.exp(1j * (2 * (jneg - nbw) + 1) * PI / nbw)) * F[nbw // 2:] / kn ** 4)
        return out, C1

    Jt, CJ1 = spline_to_matsubara(hk, dhV0.reshape(K), dhVb.reshape(K))
    J0t, _ = spline_to_matsubara(f0k, df0V0.reshape(K), df0Vb.reshape(K))
    # G(k, i k_n) on the same frequency ordering (:3309-3347)
    sig = sr.sigma(T)[:, ok]                                   # [nw, K] positive frequencies
    p = np.arange(nbw)[:, None]
    kn = (2.0 * (p - nw) + 1) * PI * T
    sigfull = np.where(p < nw, np.conj(sig[np.clip(nw - p[:, 0] - 1, 0, nw - 1)]), sig[np.clip(p[:, 0] - nw, 0, nw - 1)])
    G = T / (1j * kn - e + mu - sigfull)
    Jt = G * Jt
    chijj2_qn0 = np.sum(G * G * J0t / T, axis=0)
    Gtail = T / ((-e + mu) + 1j * (kn + sr.Sigma_inf / kn))
    G = G - Gtail
    Jt = Jt - Gtail * (-1j * CJ1 / kn)
    k0 = np.sum(G, axis=0)
    dGp = np.sum(kn * G.imag, axis=0)
    dJ0 = -np.sum(kn * Jt.imag, axis=0)
    r1, r2 = find_roots_2pol(np.ones(K, dtype=np.complex128), (-e + mu) + 0j, -sr.Sigma_inf + 0j * e)
    a1, a2 = r1 / (r1 - r2), r2 / (r2 - r1)
    b1 = CJ1 / (r1 - r2)
    b2 = -b1

    def branch(r, a, b):
        big = r.real > 0
        ex = np.where(big, np.exp(-r / T), np.exp(r / T))
        den = ex + 1.0
        fp = np.where(big, a / den, a * ex / den)
        fm = np.where(big, a * ex / den, a / den)
        fj = np.where(big, r * b * ex / den, r * b / den)
        fjb = np.where(big, r * b / den, r * b * ex / den)
        return den, fp, fm, fj, fjb

    den1, f1p, f1m, fj1, fj1b = branch(r1, a1, b1)
    den2, f2p, f2m, fj2, fj2b = branch(r2, a2, b2)
    k0 = k0 + (f1m + f2m).real
    dGm = -dGp
    dGp = dGp + (r1 * f1p + r2 * f2p).real
    dGm = dGm + (r1 * f1m + r2 * f2m).real
    dJb = -dJ0
    dJ0 = dJ0 + (fj1 + fj2).real
    dJb = dJb + (fj1b + fj2b).real
    # back to tau, analytic tails added (:3545-3620)
    Gt = np.fft.fft(G, axis=0)
    Gbeta = Gt[0].copy()
    Jtt = np.fft.ifft(Jt, axis=0) * nbw
    Jbeta = Jtt[0].copy()
    t = jj / (nbw * T)

    def tails(tt):
        e1 = np.where(r1.real > 0, np.exp(-tt * r1), np.exp((1.0 / T - tt) * r1))
        j1 = np.where(r1.real > 0, np.exp(r1 * (tt - 1.0 / T)), np.exp(r1 * tt))
        e2 = np.where(r2.real > 0, np.exp(-tt * r2), np.exp((1.0 / T - tt) * r2))
        j2 = np.where(r2.real > 0, np.exp(r2 * (tt - 1.0 / T)), np.exp(r2 * tt))
        G0t = (-a1 * e1 / den1 - a2 * e2 / den2).real
        Jinf = (b1 * j1 / den1 + b2 * j2 / den2).real
        return G0t, Jinf

    G0t, Jinf = tails(t)
    ph = np.exp(1j * (jj * PI * (nbw - 1)) / nbw)
    Gt = ph * Gt + G0t
    Jtt = Jtt / ph + Jinf
    G0b, Jinfb = tails(np.full((1, K), 1.0 / T))
    phb = np.exp(1j * PI * (nbw - 1))
    Gbeta = phb * Gbeta + G0b[0]
    Jbeta = Jbeta / phb + Jinfb[0]
    # GJ(tau) spline -> J(i q_n) (:3622-3660)
    gj = np.empty((nbw + 1, K))
    gj[:nbw] = (Gt * Jtt).real
    gj[nbw] = ((-Gt[0] - 1.0) * Jbeta).real
    d0 = (dGp * Jtt[0] + Gt[0] * dJ0).real
    dN = (dGm * Jbeta - (Gt[0] + 1.0) * dJb).real
    CJ1b = gj[0] - gj[nbw]
    a, b, c, d = clamped_spline(gj, hdt, d0, dN)
    d2J0 = 2 * b[0]
    d2Jb = 6.0 * a[nbw - 1] / (nbw * T) + 2.0 * b[nbw - 1]
    CJ3b = d2J0 - d2Jb
    J0f = np.fft.fft(6.0 * a, axis=0)
    jq = np.arange(1, nw + 1)[:, None]
    wq = 2 * jq * PI * T
    Jq = (-2.0j * CJ1b / wq + 2.0j * CJ3b / wq ** 3
          + 2.0j * ((1.0 - np.exp(-2j * jq * PI / nbw)) * J0f[1:nw + 1] / wq ** 4).imag)
    # bubble -G(tau)G(beta - tau) (:3662-3700)
    GG = np.empty((nw + 1, K))
    GG[0] = (Gt[0] * (Gt[0] + 1.0)).real
    GG[1:] = (-Gt[1:nw + 1] * Gt[nbw - np.arange(1, nw + 1)]).real
    dchi_b = dGp * (Gt[0].real + 1.0) + Gt[0].real * dGm
    a, b, c, d = clamped_spline(GG, hdt, dchi_b, np.zeros(K))
    fb = np.empty((nbw, K))
    fb[:nw] = 6.0 * a
    fb[nw:] = -fb[:nw][::-1]
    Fb = np.fft.fft(fb, axis=0)
    integ = np.sum(a * hdt ** 4 / 4.0 + b * hdt ** 3 / 3.0 + c * hdt ** 2 / 2.0 + d * hdt, axis=0)
    bub = np.empty((nw + 1, K))
    bub[0] = 2 * integ
    bub[1:] = -2.0 * dchi_b / wq ** 2 + ((1.0 - np.exp(-2j * jq * PI / nbw)) * Fb[1:nw + 1] / wq ** 4).real
    c1 = -2.0 * wt * normFact * dk * dk * bub                      # [nw + 1, K] per-k terms
    c2 = np.empty((nw + 1, K))
    c2[0] = -normFact * wt * dk * chijj2_qn0.real
    c2[1:] = -normFact * wt * dk * Jq.imag / wq
    chijj1, chijj2 = c1.sum(axis=1), c2.sum(axis=1)
    # angle bins theta_k = atan((nk0/2 - m)/(nk0/2 - l - 1)) (:3174, 3790-3796)
    theta = np.arctan((nk0 / 2 - my) / (nk0 / 2 - lx)).reshape(K)
    ib = np.floor(theta / (PI / (2.0 * ntheta))).astype(int)
    chijj1_k = np.zeros((nw + 1, ntheta))
    chijj2_k = np.zeros((nw + 1, ntheta))
    for b in range(ntheta):
        chijj1_k[:, b] = c1[:, ib == b].sum(axis=1)
        chijj2_k[:, b] = c2[:, ib == b].sum(axis=1)
    k0sum = -np.sum(2.0 * wt * normFact * d2ek[1:nbk - 1, :].reshape(K) * k0)
    # kx = 0 and kx = pi lines (:3993-4173)
    for l in (0, nbk - 1):
        mm = np.arange(nbk)
        xo2 = np.maximum(l, mm)
        yo2 = np.minimum(l, mm)
        o2 = yo2 + xo2 * (xo2 + 1) // 2
        e2 = ek[l, :]
        s2 = sr.sigma(T)[:, o2]
        sfull = np.where(p < nw, np.conj(s2[np.clip(nw - p[:, 0] - 1, 0, nw - 1)]), s2[np.clip(p[:, 0] - nw, 0, nw - 1)])
        G2 = T / (1j * kn - e2 + mu - sfull) - T / ((-e2 + mu) + 1j * (kn + sr.Sigma_inf / kn))
        kk = np.sum(G2, axis=0)
        q1, q2 = find_roots_2pol(np.ones(nbk, dtype=np.complex128), (-e2 + mu) + 0j, -sr.Sigma_inf + 0j * e2)
        aa1, aa2 = q1 / (q1 - q2), q2 / (q2 - q1)
        fm = (np.where(q1.real > 0, aa1 * np.exp(-q1 / T) / (np.exp(-q1 / T) + 1.0), aa1 / (np.exp(q1 / T) + 1.0))
              + np.where(q2.real > 0, aa2 * np.exp(-q2 / T) / (np.exp(-q2 / T) + 1.0), aa2 / (np.exp(q2 / T) + 1.0)))
        kk = kk + fm.real
        w2 = np.where((mm == 0) | (mm == nbk - 1), 1.0, 2.0)
        k0sum -= np.sum(2.0 * w2 * normFact * d2ek[l, :] * kk)
    return CondResult(chijj1, chijj2, float(k0sum.real), chijj1_k, chijj2_k)


# ----------------------------------------------------------------------------
# Aslamazov-Larkin vertex correction chijj3 (cond_opt::calc_chijj_vertex_corr_all_optim
# with chi3 = true, src/cond_opt.cpp:4292-6529)
# ----------------------------------------------------------------------------
def al_frequencies(nbw: int, mmin: int) -> np.ndarray:
    """The non-uniform bosonic grid of the AL term (src/cond_opt.cpp:5123-5155):
    every n up to (N0-1)/2^mmin, then mmin blocks of (N0-1)/2^(mmin+1) points
    whose spacing doubles per block (N0 = nbw/2 + 1)."""
    N0 = nbw // 2 + 1
    jf = (N0 - 1) // (2 ** mmin)
    Nj = (N0 - 1) // (2 ** (mmin + 1))
    out = list(range(jf + 1))
    n, d = jf, 1
    for _ in range(mmin):
        d *= 2
        for _ in range(Nj):
            n += d
            out.append(n)
    return np.array(out, dtype=np.int64)


@dataclass
class ALResult:
    ind_freq: np.ndarray  # [N] the bosonic indices n of the grid
    chijj3: np.ndarray    # [N] AL correction chi_jj3(iq_n); entry 0 is not computed (0)
    chijj3_k: np.ndarray  # [N, ntheta] angle-resolved


def conductivity_al(sv: Solve, tp, tpp, t3, U, T, mmin=3, ntheta=1) -> ALResult:
    """The AL branch of cond_opt::calc_chijj_vertex_corr_all_optim
    (src/cond_opt.cpp:4292-6420), vectorised over the K4 grid of interior kx
    points; the per-frequency loop follows the reference's order."""
    nk0, nbw = sv.nk0, sv.Nw0
    nbk = nk0 // 2 + 1
    nw = nbw // 2
    ek = dispersion(nbk, tp, tpp, t3)
    er = hopping_octant(nbk, tp, tpp, t3)
    mu0, mu = sv.mu0, sv.mu
    sr, c0 = sv.sigma, sv.chi0
    Usp, Uch = sv.U.Usp, sv.U.Uch
    normFact = 1.0 / (nk0 * nk0)
    kq = np.arange(nbk) * PI / (nbk - 1)
    dek = grad_ek_x(kq[1:nbk - 1, None], kq[None, :], tp, tpp, t3)              # [nbk-2, nbk]
    xk = ek[1:nbk - 1, :] - mu0
    pos = xk > 0
    K = (nbk - 2) * nbk
    lx = np.arange(1, nbk - 1)[:, None] * np.ones((1, nbk), dtype=int)
    my = np.ones((nbk - 2, 1), dtype=int) * np.arange(nbk)[None, :]
    xo, yo = np.maximum(lx, my), np.minimum(lx, my)
    oidx = yo + xo * (xo + 1) // 2                                              # r = (l+1, m) in the octant
    ok = oidx.reshape(K)
    # h(r, tau_j) and its tau-derivatives at 0 and beta (:4304-4330, :2744-2783)
    h = np.empty((nbw + 1, nbk - 2, nbk))
    for j in range(nbw + 1):
        t = j / (T * nbw)
        h[j] = dst_dct(np.where(pos, normFact * dek * np.exp(-xk * t) / (np.exp(-xk / T) + 1.0),
                                normFact * dek * np.exp(xk * (1.0 / T - t)) / (np.exp(xk / T) + 1.0)))
    dh0 = dst_dct(np.where(pos, -normFact * dek * xk / (np.exp(-xk / T) + 1.0),
                           -normFact * dek * xk * np.exp(xk / T) / (np.exp(xk / T) + 1.0)))
    dhb = dst_dct(np.where(pos, -normFact * dek * xk * np.exp(-xk / T) / (np.exp(-xk / T) + 1.0),
                           -normFact * dek * xk / (np.exp(xk / T) + 1.0)))
    # G(r, -tau_j) = DCT-I[G0(k, -tau_j)] / L^2 and its tau-derivative at 0 and beta (:4382-4446)
    ekm = ek - mu0
    neg = ek < mu0
    Grt = np.empty((nbw + 1, nbk * (nbk + 1) // 2))
    for j in range(nbw + 1):
        t = j / (T * nbw)
        fr = np.where(neg, normFact * np.exp(ekm * t) / (np.exp(ekm / T) + 1.0),
                      normFact * np.exp(ekm * (t - 1.0 / T)) / (np.exp(-ekm / T) + 1.0))
        Grt[j] = to_octant(dct2(fr))
    dG0 = to_octant(dct2(np.where(neg, normFact * ekm / (np.exp(ekm / T) + 1.0),
                                  normFact * ekm * np.exp(-ekm / T) / (np.exp(-ekm / T) + 1.0))))
    dGb = er.copy()
    dGb[0] = -mu0
    dGb = dGb - dG0
    # h G in q space and its spline over tau -> hG(q, i q_n) (:5158-5330)
    dhG0 = dst_dct(dh0 * Grt[0][oidx] + h[0] * dG0[oidx]).reshape(K)
    dhGb = dst_dct(dhb * Grt[nbw][oidx] + h[nbw] * dGb[oidx]).reshape(K)
    hG = np.empty((nbw + 1, K))
    for j in range(nbw + 1):
        hG[j] = dst_dct(h[j] * Grt[j][oidx]).reshape(K)
    hdt = 1.0 / (nbw * T)
    a, b, c, d = clamped_spline(hG, hdt, dhG0, dhGb)
    F = np.fft.fft(6.0 * a, axis=0)
    integ = np.sum(a * hdt ** 4 / 4.0 + b * hdt ** 3 / 3.0 + c * hdt ** 2 / 2.0 + d * hdt, axis=0)
    hq = np.empty((nw, K))
    hq[0] = 2 * integ
    jq = np.arange(1, nw)[:, None]
    hq[1:] = 2 * ((1.0 - np.exp(-2j * jq * PI / nbw)) * F[1:nw]).real
    hg2 = 2 * (dhG0 - dhGb)
    chiq = c0.chiqw[:, ok]                                                      # [nw+1, K]
    cinf, cinf2 = c0.chi0_inf[ok], c0.chi0_inf2[ok]

    def chi0_at(p):
        p = np.abs(p)
        wn = 2 * PI * p * T
        if p <= nw:
            return chiq[p]
        return cinf / wn ** 2 + cinf2 / wn ** 4

    def hg_at(p):
        p = abs(p)
        wn = 2 * PI * p * T
        if p == 0:
            return hq[0]
        return -hg2 / wn ** 2 + hq[min(p, nw - 1)] / wn ** 4

    ind_freq = al_frequencies(nbw, mmin)
    N = ind_freq.size
    chijj3 = np.zeros(N)
    chijj3_k = np.zeros((N, ntheta))
    e = ek[1:nbk - 1, :].reshape(K)
    dk = dek.reshape(K)
    wt = np.where((my == 0) | (my == nbk - 1), 2.0, 4.0).reshape(K)
    theta = np.arctan((nk0 / 2 - my) / (nk0 / 2 - lx)).reshape(K)
    ib = np.floor(theta / (PI / (2.0 * ntheta))).astype(int)
    C2, C3 = sr.Sigma_inf2[ok], sr.Sigma_inf3[ok]
    Sk = sr.S[:, ok]                                                            # [nw, K] 1/z^4 coefficient
    jj = np.arange(nbw)[:, None]
    zsp0 = 1j * np.sqrt(Usp * cinf / 2.0)
    zsp1 = -zsp0
    zch0 = np.sqrt(Uch * cinf / 2.0) + 0j
    zch1 = -zch0

    for n in range(1, N):
        nn = int(ind_freq[n])
        qn = 2.0 * nn * PI * T
        nc = nn // 2
        # I_n(q, i q_m): the difference quotient of hG against chi0 (:5351-5493)
        # at q_m = -q_n/2 (n even) both ends of the quotient meet: the
        # reference extrapolates from the two previous m, (4 D(m-1) - D(m-2))/3
        HG = np.empty((nbw, K))
        D1 = np.zeros(K)
        D2 = np.zeros(K)
        for j in range(nbw):
            first = j < nw - nc
            p1, p2 = (j, j + nn) if first else (j - nbw, j - nbw + nn)
            ch1 = chi0_at(p1)
            pre = 3 * Usp * ch1 / (1.0 - Usp * ch1 / 2) + Uch * ch1 / (1.0 + Uch * ch1 / 2)
            if not first and nn % 2 == 0 and j - nbw == -(nn // 2):
                HG[j] = pre * (4 * D1 - D2) / 3.0
                continue
            q = (hg_at(p1) - hg_at(p2)) / (ch1 - chi0_at(p2))
            if not first and nn % 2 == 0:
                D2, D1 = D1, q
            HG[j] = pre * q
        # to tau: minus the asymptote, FFT, plus its closed form (:5500-5622)
        wn = np.where(jj < nw - nc, 2 * jj * PI * T, 2 * (jj - nbw) * PI * T)
        cq = -cinf
        Hinf = hg2 * (3.0 * Usp / (-wn * wn - Usp * cq / 2.0) + Uch / (-wn * wn + Uch * cq / 2.0))
        ft = T * (HG - Hinf)
        dtauH0 = -np.sum(wn * ft, axis=0)
        ft = np.fft.fft(ft, axis=0)
        tt = jj / (nbw * T)
        tmp_sp = (np.exp(-zsp0 * tt) / ((np.exp(-zsp0 / T) - 1.0) * (zsp0 - zsp1))
                  + np.exp(-zsp1 * tt) / ((np.exp(-zsp1 / T) - 1.0) * (zsp1 - zsp0)))
        tmp_ch = (np.exp(-zch0 * tt) / ((np.exp(-zch0 / T) - 1.0) * (zch0 - zch1))
                  + np.exp(zch1 * (1.0 / T - tt)) / ((1.0 - np.exp(zch1 / T)) * (zch1 - zch0)))
        Hq = np.empty((nbw + 1, K), dtype=np.complex128)
        Hq[:nbw] = ft + hg2 * (3.0 * Usp * tmp_sp + Uch * tmp_ch)
        tsp = (1.0 / ((1.0 - np.exp(zsp0 / T)) * (zsp0 - zsp1)) + 1.0 / ((1.0 - np.exp(zsp1 / T)) * (zsp1 - zsp0)))
        tch = (np.exp(-zch0 / T) / ((np.exp(-zch0 / T) - 1.0) * (zch0 - zch1))
               + 1.0 / ((1.0 - np.exp(zch1 / T)) * (zch1 - zch0)))
        Hq[nbw] = ft[0] + hg2 * (3.0 * Usp * tsp + Uch * tch)
        tsp = (-zsp0 / ((np.exp(-zsp0 / T) - 1.0) * (zsp0 - zsp1)) - zsp1 / ((np.exp(-zsp1 / T) - 1.0) * (zsp1 - zsp0)))
        tch = (-zch0 / ((np.exp(-zch0 / T) - 1.0) * (zch0 - zch1))
               - zch1 * np.exp(zch1 / T) / ((1.0 - np.exp(zch1 / T)) * (zch1 - zch0)))
        dH0 = 1j * dtauH0 + hg2 * (3.0 * Usp * tsp + Uch * tch)
        tsp = (-zsp0 * np.exp(-zsp0 / T) / ((np.exp(-zsp0 / T) - 1.0) * (zsp0 - zsp1))
               - zsp1 * np.exp(-zsp1 / T) / ((np.exp(-zsp1 / T) - 1.0) * (zsp1 - zsp0)))
        tch = (-zch0 * np.exp(-zch0 / T) / ((np.exp(-zch0 / T) - 1.0) * (zch0 - zch1))
               - zch1 / ((1.0 - np.exp(zch1 / T)) * (zch1 - zch0)))
        dHb = 1j * dtauH0 + hg2 * (3.0 * Usp * tsp + Uch * tch)

        def dd(z):
            """DST x DCT of the real and imaginary parts (q -> r or r -> k)."""
            z = z.reshape(z.shape[:-1] + (nbk - 2, nbk))
            return (dst_dct(z.real) + 1j * dst_dct(z.imag)).reshape(z.shape[:-2] + (K,))

        # q -> r (:5628-5716), then the mirror H2(tau) = H(beta - tau) (:5718-5727)
        Hr = dd(normFact * Hq)
        dH0r, dHbr = dd(normFact * dH0), dd(normFact * dHb)
        H2r = Hr[::-1]
        dH20r, dH2br = -dHbr, -dH0r
        Gk = Grt[:, ok]                                                         # G(r, -tau_j) on the K4 r grid
        dG0k, dGbk = dG0[ok], dGb[ok]

        def to_k(Hr_, d0r, dbr):
            """times G(r, -tau) and DST x DCT back to k (:5729-5900)."""
            d0 = dd(Hr_[0].real * dG0k + d0r.real * Gk[0]) + 1j * dd(Hr_[0].imag * dG0k + d0r.imag * Gk[0])
            db = (dd(Hr_[nbw].real * dGbk + dbr.real * Gk[nbw])
                  + 1j * dd(Hr_[nbw].imag * dGbk + dbr.imag * Gk[nbw]))
            Hk = dd(Hr_.real * Gk) + 1j * dd(Hr_.imag * Gk)
            return Hk, d0, db

        Hk, d0k, dbk = to_k(Hr, dH0r, dHbr)
        H2k, d20k, d2bk = to_k(H2r, dH20r, dH2br)

        def to_matsubara(Hk_, d0, db):
            """two splines (Re, Im) over tau, pre-twiddled FFT (:5906-5985)."""
            ar, br, _, _ = clamped_spline(Hk_.real, hdt, d0.real, db.real)
            ai, bi, _, _ = clamped_spline(Hk_.imag, hdt, d0.imag, db.imag)
            d2S0 = 2 * br[0] + 1j * 2 * bi[0]
            d2Sb = (6.0 * ar[nbw - 1] / (nbw * T) + 2.0 * br[nbw - 1]
                    + 1j * (6.0 * ai[nbw - 1] / (nbw * T) + 2.0 * bi[nbw - 1]))
            ph = np.exp(-1j * PI * jj / nbw)
            Fq = np.fft.fft(ph * 6.0 * ar + 1j * ph * 6.0 * ai, axis=0)
            return Fq, Hk_[0] + Hk_[nbw], d0 + db, d2S0 + d2Sb

        F1, cw1, dsum1, d2sum1 = to_matsubara(Hk, d0k, dbk)
        F2, cw2, dsum2, d2sum2 = to_matsubara(H2k, d20k, d2bk)
        HGf = np.empty((nbw, K), dtype=np.complex128)
        HG2f = np.empty((nbw, K), dtype=np.complex128)
        for j in range(nbw):
            if j < nw - nc:
                w1 = (2 * (j + nn) + 1) * PI * T
                idx = j + nn if j + nn < nbw else None
            else:
                w1 = (2 * (j + nn - nbw) + 1) * PI * T
                if j + nn - nbw < 0:
                    idx = j + nn
                elif j + nn - nbw < nbw:
                    idx = j + nn - nbw
                else:
                    idx = None
            v = -1j * cw1 / w1 - dsum1 / w1 ** 2 + 1j * d2sum1 / w1 ** 3
            if idx is not None:
                v = v + (1.0 - np.exp(-1j * (2 * (j + nn) + 1) * PI / nbw)) * F1[idx] / w1 ** 4
            HGf[j] = v
            w2 = (2 * j + 1) * PI * T if j < nw - nc else (2 * (j - nbw) + 1) * PI * T
            HG2f[j] = (-1j * cw2 / w2 - dsum2 / w2 ** 2 + 1j * d2sum2 / w2 ** 3
                       + (1.0 - np.exp(-1j * (2 * j + 1) * PI / nbw)) * F2[j] / w2 ** 4)

        # accumulate with G(k, i k_j) G(k, i k_{j+n}) (:6253-6398)
        def green(f):
            """G(k, i k_f) for the fermionic index f (k_f = (2f+1) pi T, any sign)."""
            kn = (2 * f + 1) * PI * T
            if f >= 0:
                s = (-C2 / kn ** 2 + 1j * (-sr.Sigma_inf / kn + C3 / kn ** 3))
                if f < nw:
                    s = s + Sk[f] / kn ** 4
            else:
                s = (-C2 / kn ** 2 + 1j * (-sr.Sigma_inf / kn + C3 / kn ** 3))
                if -f - 1 < nw:
                    s = s + np.conj(Sk[-f - 1]) / kn ** 4
            return 1.0 / (1j * kn - e + mu - s)

        acc = np.zeros(K, dtype=np.complex128)
        for j in range(nbw):
            f1 = j if j < nw - nc else j - nbw
            acc += green(f1) * green(f1 + nn) * (HGf[j] - HG2f[j])
        term = -1j * U * T * normFact * wt * dk * acc / (2 * qn)
        chijj3[n] = term.real.sum()
        for b in range(ntheta):
            chijj3_k[n, b] = term.real[ib == b].sum()
    return ALResult(ind_freq, chijj3, chijj3_k)


# ----------------------------------------------------------------------------
# spin correlation length (chi::sp_corr_length, src/chi.cpp:450-718) with the
# Fermi velocity at the hot spots (chi::vF_hot_spots, src/chi.cpp:420-447) on
# the non-interacting Fermi surface (green0::find_FS, src/green0.cpp:626-676)
# ----------------------------------------------------------------------------
def dispk(kx, ky, tp, tpp, t3):
    """hamiltonien::dispk (src/hamiltonien.cpp:119-122), scalar, libm cos (NaN
    for a non-finite argument, as C's cos)."""

    def c(x):
        return math.cos(x) if math.isfinite(x) else math.nan

    return (-2.0 * (c(kx) + c(ky)) - 4.0 * tp * c(kx) * c(ky) - 2.0 * tpp * (c(2 * kx) + c(2 * ky))
            - 4 * t3 * (c(2 * kx) * c(ky) + c(2 * ky) * c(kx)))


def find_fs(mu0, tp, tpp, t3, nk=10001):
    """green0::find_FS(nk): on each line kx - ky = kx0, kx0 = j pi/(nk-1), the
    root kx in [kx0, pi] of eps(kx, kx - kx0) - mu0 by the bounded find_zero
    from init {(kx0 + pi)/2, kx0, pi}; stops at the first line without a root.
    Returns the list of (kx, ky); lines after a failure are absent."""
    fs = []
    for j in range(nk):
        kx0 = j * PI / (nk - 1)
        init = (0.5 * (kx0 + PI), kx0, PI)
        try:
            root, _ = find_zero(lambda kx: dispk(kx, kx - kx0, tp, tpp, t3) - mu0, init, lims=(kx0, PI))
        except RootNotFound:
            break
        fs.append((root, root - kx0))
    return fs


def vf_hot_spots(fs, tp, tpp, t3, nk=10001):
    """chi::vF_hot_spots: first pair of consecutive Fermi-surface points whose
    kx + ky - pi changes sign (or the last pair), |grad eps| at their midpoint.
    Points of lines without a root read as (-1, -1), as the reference's array."""
    pts = list(fs) + [(-1.0, -1.0)] * (nk - len(fs))
    kx1, ky1 = pts[0]
    kx2, ky2 = pts[1]
    j = 1
    while (kx1 + ky1 - PI) * (kx2 + ky2 - PI) > 0 and j < nk - 1:
        j += 1
        kx1, ky1 = kx2, ky2
        kx2, ky2 = pts[j]
    kx, ky = (kx1 + kx2) / 2, (ky1 + ky2) / 2
    s, c = math.sin, math.cos
    gx = 2.0 * s(kx) + 4.0 * tp * s(kx) * c(ky) + 4.0 * tpp * s(2 * kx) + 4 * t3 * (2.0 * s(2 * kx) * c(ky) + c(2 * ky) * s(kx))
    gy = 2.0 * s(ky) + 4.0 * tp * c(kx) * s(ky) + 4.0 * tpp * s(2 * ky) + 4 * t3 * (c(2 * kx) * s(ky) + 2.0 * s(2 * ky) * c(kx))
    return math.sqrt(gx * gx + gy * gy)


def sp_corr_length(chi0_q0, chi0max, qmax, Usp, nbq, mu0, tp, tpp, t3, nk_fs=10001):
    """chi::sp_corr_length: the spin correlation lengths along y and x from the
    half maximum of chi_sp(q, 0) = chi0/(1 - Usp chi0/2) around qmax on the
    lattice, and from the asymptotic (Ornstein-Zernike) form with the second
    difference of chi0 at qmax; vF from vF_hot_spots.  chi0_q0 is chi0(q, 0) in
    the octant layout m + l(l+1)/2.  Returns dict vF, xi_y, xi_x, xiAs_y,
    xiAs_x, xi0_y, xi0_x."""
    vF = vf_hot_spots(find_fs(mu0, tp, tpp, t3, nk_fs), tp, tpp, t3, nk_fs)
    a = np.asarray(chi0_q0, dtype=np.float64)

    def csp(i):
        return a[i] / (1.0 - Usp * a[i] / 2.0)

    def oi(x, y):
        return y + (x * (x + 1)) // 2

    q0x, q1x = int(qmax[0]), int(qmax[1])
    dq = PI / (nbq - 1)
    half = chi0max / (1.0 - Usp * chi0max / 2.0) / 2.0
    # along y at kx = qmax_x
    l, m = q0x, 0
    base = (l * (l + 1)) // 2
    cur = csp(base)
    prev = cur
    while cur < half and m <= q1x:
        m += 1
        prev = cur
        cur = csp(base + m)
    q0 = (m - 1) * dq
    qHM = dq * (half - prev) / (cur - prev) + q0
    xi_y = 1.0 / (q1x * dq - qHM)
    # along x at ky = qmax_y, from the diagonal
    m = q1x
    l = m
    cur = csp(oi(l, m))
    if cur < half:
        while cur < half and l <= q0x:
            l += 1
            prev = cur
            cur = csp(oi(l, m))
        q0 = (l - 1) * dq
        qHM = dq * (half - prev) / (cur - prev) + q0
        xi_x = 1.0 / (q0x * dq - qHM)
    else:
        xi_x = xi_y
    # asymptotic form
    fac = (nbq - 1) * (nbq - 1) / (PI * PI)
    if q0x == nbq - 1 and q1x == nbq - 1:
        dchi2 = 2.0 * (a[base + nbq - 2] - chi0max) * fac
        xi0_x = math.sqrt(-0.5 * dchi2 / chi0max)
        xiAs_x = xi0_x * math.sqrt(Usp / (2.0 / chi0max - Usp))
        xi0_y, xiAs_y = xi0_x, xiAs_x
    else:
        x, y = q0x, q1x - 1
        if y < 0:
            y = q1x + 1
        cl = a[oi(x, y)]
        y = q1x
        cm = a[oi(x, y)]
        y = q1x + 1
        if y > x:
            x, y = q1x + 1, q0x
        cr = a[oi(x, y)]
        dchi2 = (cr - 2 * cm + cl) * fac
        xi0_y = math.sqrt(-0.5 * dchi2 / chi0max)
        xiAs_y = xi0_y * math.sqrt(Usp / (2.0 / chi0max - Usp))
        x, y = q0x - 1, q1x
        if y > x:
            x, y = q1x, q0x - 1
            if y < 0:
                y = q0x + 1
        cl = a[oi(x, y)]
        x, y = q0x, q1x
        cm = a[oi(x, y)]
        x = q0x + 1
        if x > nbq - 1:
            x = q0x - 1
        cr = a[oi(x, y)]
        dchi2 = (cr - 2 * cm + cl) * fac
        xi0_x = math.sqrt(-0.5 * dchi2 / chi0max)
        xiAs_x = xi0_x * math.sqrt(Usp / (2.0 / chi0max - Usp))
    return dict(vF=vF, xi_y=xi_y, xi_x=xi_x, xiAs_y=xiAs_y, xiAs_x=xiAs_x, xi0_y=xi0_y, xi0_x=xi0_x)
