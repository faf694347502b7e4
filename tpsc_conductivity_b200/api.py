"""Python mirror of the reference's TPSC class interface over the C ABI.

``Green(nk0, Nw0, n, T, eta, params)`` takes the arguments of the reference's
``green`` constructor (src/green.h:26; params = {tp, tpp, t3, U}) and offers
its hot-path methods under the same names: ``calc_chiqw_FFT_spline``,
``find_Usp_Uch``, ``calc_chirt``, ``calc_Self_FFT_spline``, ``traceSelfG``,
``find_mu``, ``traceSelfG2``, ``traceChi0``.  Results come back as numpy
arrays in the reference's layouts (octant index m + l(l+1)/2, frequency
major).  Every computation runs in the CUDA library; a missing library or
device raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


class Context:
    """One CUDA stream and the device arrays of every grid it has used."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        st = C.c_int(0)
        self.h = self.lib.tpsc_create(device, C.byref(st))
        if not self.h:
            raise _lib.TPSCError(st.value, self.lib.tpsc_last_error(None).decode())

    def call(self, name, *args):
        _lib.check(self.lib, self.h, getattr(self.lib, name)(self.h, *args))

    def close(self):
        if getattr(self, "h", None):
            self.lib.tpsc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Green:
    """Drop-in for the reference's ``green`` object on the TPSC hot path."""

    def __init__(self, nk0=8, Nw0=32, n=1.0, T=1.0, eta=0.1, params=None, device=0, ctx=None):
        tp, tpp, t3, U = (params if params is not None else (0.0, 0.0, 0.0, 1.0))
        self.nk0, self.Nw0, self.density, self.tem, self.eta = nk0, Nw0, n, T, eta
        self.tp, self.tpp, self.t3, self.U = tp, tpp, t3, U
        self.ctx = ctx or Context(device)
        self.ctx.call("tpsc_set_model", nk0, Nw0, n, T, tp, tpp, t3, U)

    def set_form(self, form):
        """Root-search form of the context: _lib.FORM_REFERENCE (the reference's
        find_zero) or _lib.FORM_NEWTON (safeguarded Newton)."""
        self.ctx.call("tpsc_set_form", int(form))

    def set_graph_mode(self, mode):
        """CUDA graphs for Newton-form solves of the context: 0 off, 1 replay a
        repeated solve (default), 2 capture every solve."""
        self.ctx.call("tpsc_set_graph_mode", int(mode))

    def graph_stats(self):
        """{captures, replays, kernels per graph, off} of the context's solve graph."""
        out = np.zeros(4, dtype=np.int64)
        self.ctx.call("tpsc_graph_stats", out.ctypes.data_as(C.c_void_p))
        return dict(zip(("captures", "replays", "kernels", "off"), out.tolist()))

    # ---- stages (reference method names) ---------------------------------
    def calc_chiqw_FFT_spline(self, nq0=None, nw0=None):
        """chi0::calc_chiqw_FFT_spline (src/chi0.cpp:279)."""
        self.ctx.call("tpsc_chi0", nq0 or self.nk0, nw0 or self.Nw0)

    def traceChi0(self):
        """chi0::traceChi0 (src/chi0.cpp:1498): (raw, extrapolated)."""
        out = np.zeros(2)
        self.ctx.call("tpsc_trace_chi0", _dptr(out))
        return float(out[0]), float(out[1])

    def traceDiffChi(self, channel, Uv):
        """traceDiffChispChi0 (channel 0) / traceDiffChichChi0 (channel 1), src/chi.cpp:738-830."""
        t, dt = C.c_double(), C.c_double()
        self.ctx.call("tpsc_trace_diff_chi", channel, Uv, C.byref(t), C.byref(dt))
        return t.value, dt.value

    def find_Usp_Uch_grid(self, nq0, nw0):
        """chi::find_Usp_Uch(nq0, nw0, Usc) (src/chi.cpp:846)."""
        out = np.zeros(2)
        self.ctx.call("tpsc_find_Usp_Uch_grid", nq0, nw0, _dptr(out))
        return float(out[0]), float(out[1])

    def find_Usp_Uch(self):
        """chi::find_Usp_Uch() (src/chi.cpp:210): half grid, full grid, dblOcc."""
        self.ctx.call("tpsc_find_Usp_Uch")

    def sp_corr_length(self):
        """chi::sp_corr_length (src/chi.cpp:450-718) after find_Usp_Uch: the Fermi
        velocity at the hot spots and the spin correlation lengths (half maximum
        of chi_sp(q, 0) along y and x, asymptotic form, xi0)."""
        out = np.zeros(7)
        self.ctx.call("tpsc_sp_corr_length", _dptr(out))
        return dict(zip(["vF", "xi_y", "xi_x", "xiAs_y", "xiAs_x", "xi0_y", "xi0_x"], out.tolist()))

    def sumrule_tangents(self):
        """d(Usp, Uch, D)/d(U, mu, t') on the current grid after its chi0 and
        roots (forward tangents; mu a shift of mu0 at fixed n, t' at fixed n).
        Returns a dict of dicts: J[param][output]."""
        out = np.zeros(9)
        self.ctx.call("tpsc_sumrule_tangents", _dptr(out))
        return {p: {k: float(out[3 * i + j]) for j, k in enumerate(("Usp", "Uch", "D"))}
                for i, p in enumerate(("U", "mu", "tp"))}

    def sumrule_vjp(self, cot):
        """The backward pair: sum_k cot[k] d(Usp, Uch, D)_k/d(U, mu, t')."""
        c = np.asarray(cot, dtype=np.float64)
        g = np.zeros(3)
        self.ctx.call("tpsc_sumrule_vjp", _dptr(c), _dptr(g))
        return g

    def set_mu_shift(self, dmu):
        """mu0 = density root + dmu on every grid from the next stage on."""
        self.ctx.call("tpsc_set_mu_shift", float(dmu))

    def calc_chirt(self):
        """chi::calc_chirt (src/chi.cpp:37)."""
        self.ctx.call("tpsc_vertex")

    def calc_self_energy(self):
        """green::calc_Self_FFT_spline after calc_chirt (src/green.cpp:1741-2025)."""
        self.ctx.call("tpsc_self_energy")

    def calc_Self_FFT_spline(self):
        """green::calc_Self_FFT_spline (src/green.cpp:1673): find_Usp_Uch (two
        grids), calc_chirt, then the self-energy."""
        self.find_Usp_Uch()
        self.calc_chirt()
        self.calc_self_energy()

    def traceSelfG(self):
        """green::traceSelfG (src/green.cpp:3001): (sum, sum with asymptotic correction)."""
        out = np.zeros(2)
        self.ctx.call("tpsc_trace_self_G", _dptr(out))
        return float(out[0]), float(out[1])

    def traceDiffG(self, mu, derivative=False):
        """green::traceDiffG (src/green.cpp:3108); with derivative=True also
        d Tr(G - G0)/d mu from the same pass."""
        t, dt = C.c_double(), C.c_double()
        self.ctx.call("tpsc_trace_diff_G", mu, C.byref(t), C.byref(dt))
        return (t.value, dt.value) if derivative else t.value

    def find_mu(self):
        """green::find_mu (src/green.cpp:3185), followed by traceSelfG2."""
        self.ctx.call("tpsc_find_mu")

    def solve(self):
        """One full TPSC solve on the model grid (no half-grid pre-pass)."""
        self.ctx.call("tpsc_solve")

    # ---- results ----------------------------------------------------------
    def scalars(self) -> dict:
        out = np.zeros(len(_lib.SCALARS))
        self.ctx.call("tpsc_get_scalars", _dptr(out), len(out))
        return dict(zip(_lib.SCALARS, out.tolist()))

    def dims(self):
        d = (C.c_int * 4)()
        self.ctx.call("tpsc_get_dims", d)
        return tuple(d)

    def ek(self):
        nk0, nw0, nbk, n8 = self.dims()
        out = np.zeros(nbk * nbk)
        self.ctx.call("tpsc_get_ek", _dptr(out))
        return out.reshape(nbk, nbk)

    def chi0(self, full=True):
        nk0, nw0, nbk, n8 = self.dims()
        nb = nw0 // 2 + 1
        cq = np.zeros((nb, n8)) if full else None
        ci, ci2, dc = np.zeros(n8), np.zeros(n8), np.zeros(n8)
        self.ctx.call("tpsc_get_chi0", _dptr(cq), _dptr(ci), _dptr(ci2), _dptr(dc))
        return dict(chiqw=cq, chi0_inf=ci, chi0_inf2=ci2, dtau_chirt0=dc)

    def vertex(self):
        nk0, nw0, nbk, n8 = self.dims()
        out = np.zeros((nw0 // 2 + 1, n8))
        self.ctx.call("tpsc_get_vertex", _dptr(out))
        return out

    def self_energy(self, out=None):
        """S (coefficient of 1/z^4) as complex [Nw0/2, N8] plus Sigma_inf2/3/4."""
        nk0, nw0, nbk, n8 = self.dims()
        if out is None:
            out = np.zeros((nw0 // 2, n8), dtype=np.complex128)
        s2, s3, s4 = np.zeros(n8), np.zeros(n8), np.zeros(n8)
        self.ctx.call("tpsc_get_self", _dptr(out.view(np.float64)), _dptr(s2), _dptr(s3), _dptr(s4))
        return dict(S=out, Sigma_inf2=s2, Sigma_inf3=s3, Sigma_inf4=s4)

    def self_energy_async(self, out, s2=None, s3=None, s4=None):
        """The arrays of self_energy() copied to the host without waiting
        (tpsc_get_self_async): ``out`` complex [Nw0/2, N8] (and the optional
        float64 [N8] arrays) must stay alive, and should be pinned for the copy
        to overlap the next stages; read them after wait_copies()."""
        self.ctx.call("tpsc_get_self_async", _dptr(out.view(np.float64)), _dptr(s2), _dptr(s3), _dptr(s4))

    def sigma_async32(self, out):
        """The full Sigma(k, i w_n), n < Nw0/2, formed in FP64 on the device and
        copied to the host in FP32 without waiting (tpsc_get_sigma32_async):
        ``out`` complex64 [Nw0/2, N8], half the bytes of S over the host link;
        the mixed-precision form's result in its own precision.  Read after
        wait_copies()."""
        out = np.asarray(out)
        if out.dtype != np.complex64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous complex64 array")
        self.ctx.call("tpsc_get_sigma32_async", out.ctypes.data_as(C.c_void_p))

    def wait_copies(self, join_stream=False):
        """Waits for the copies of self_energy_async (or, with join_stream, makes
        the context stream wait for them)."""
        self.ctx.call("tpsc_wait_copies", 1 if join_stream else 0)

    def sigma(self):
        """Full Sigma(k, i w_n), n < Nw0/2 (src/green.cpp:3039)."""
        r = self.self_energy()
        sc = self.scalars()
        nj = r["S"].shape[0]
        z = 1j * (2 * np.arange(nj)[:, None] + 1) * np.pi * self.tem
        return (sc["Sigma_inf"] / z + r["Sigma_inf2"] / z ** 2 + r["Sigma_inf3"] / z ** 3
                + r["S"] / z ** 4)

    def pade_sigma(self, z, n_idx=None, Nn=10, mode=0):
        """Sigma(k, z) and A(k, z) at complex energies z for every octant k, from
        Nn Matsubara samples (mode 0 Pade, 1 Lagrange polynomial), as
        green::MDC / find_FS_inter do (src/green.cpp:814-1068, 2210-2341)."""
        nk0, nw0, nbk, n8 = self.dims()
        z = np.ascontiguousarray(np.atleast_1d(np.asarray(z, dtype=np.complex128)))
        idx = np.ascontiguousarray(np.arange(Nn) if n_idx is None else np.asarray(n_idx), dtype=np.int32)
        sig = np.zeros((n8, z.size), dtype=np.complex128)
        A = np.zeros((n8, z.size))
        self.ctx.call("tpsc_pade_sigma", idx.ctypes.data_as(C.POINTER(C.c_int)), int(idx.size),
                      _dptr(z.view(np.float64)), int(z.size), int(mode), _dptr(sig.view(np.float64)), _dptr(A))
        return sig, A

    def Gwn_local(self):
        """green::Gwn_local (src/green.cpp:209): local G(i w_n), n < Nw0/2."""
        nk0, nw0, nbk, n8 = self.dims()
        out = np.zeros(nw0 // 2, dtype=np.complex128)
        self.ctx.call("tpsc_gwn_local", _dptr(out.view(np.float64)))
        return out

    def stage_times(self):
        out = np.zeros(8)
        self.ctx.call("tpsc_stage_times", _dptr(out), 8)
        return dict(zip(["chi0", "sumrules", "vertex", "self", "mu", "cond_slices", "cond_tau", "cond_finish"],
                        out.tolist()))


class CondOpt(Green):
    """Drop-in for the reference's ``cond_opt`` (src/cond_opt.h:25), a ``green``
    with the current-current correlator."""

    def __init__(self, nk0=8, Nw0=32, n=1.0, T=1.0, eta=0.1, params=None, device=0, ctx=None):
        super().__init__(nk0, Nw0, n, T, eta, params, device, ctx)

    def calc_chijj_vertex_corr_all_optim(self, chi3=False, mmin=3, N_theta_k=1, k_chijj=None, nk_chijj=0):
        """cond_opt::calc_chijj_vertex_corr_all_optim (src/cond_opt.cpp:2537-6529):
        the bubble and the Maki-Thompson correction, and with ``chi3`` the
        Aslamazov-Larkin correction on the non-uniform grid of ``mmin``.
        Computes Sigma and mu first when they are missing, as the reference
        does (src/cond_opt.cpp:2550-2560).  ``k_chijj`` and ``nk_chijj`` do not
        change chi_jj in the reference and are accepted for the signature's
        sake.  Returns chijj1, chijj2 [Nw0/2+1], kx0, the angle-resolved
        chijj1_k, chijj2_k [Nw0/2+1, N_theta_k] and, with ``chi3``, the AL
        grid ind_freq [N], chijj3 [N] and chijj3_k [N, N_theta_k]."""
        self._nbins = int(N_theta_k)
        try:
            self.ctx.call("tpsc_chijj", int(N_theta_k))
        except _lib.TPSCError as e:
            if e.status != 5:
                raise
            self.calc_Self_FFT_spline()
            self.traceSelfG()
            self.find_mu()
            self.ctx.call("tpsc_chijj", int(N_theta_k))
        out = self.chijj()
        if chi3:
            self.ctx.call("tpsc_chijj3", int(mmin), int(N_theta_k))
            out.update(self.chijj3())
        return out

    def chijj3(self):
        """Results of the last Aslamazov-Larkin evaluation: the grid ind_freq,
        chijj3 and the angle-resolved chijj3_k."""
        n = np.zeros(1, dtype=np.int32)
        self.ctx.call("tpsc_get_chijj3", 0, n.ctypes.data_as(_lib._ip), None, None, None)
        N = int(n[0])
        nb = getattr(self, "_nbins", 1)
        ind = np.zeros(N, dtype=np.int32)
        c3, k3 = np.zeros(N), np.zeros(N * nb)
        self.ctx.call("tpsc_get_chijj3", N, n.ctypes.data_as(_lib._ip), ind.ctypes.data_as(_lib._ip), _dptr(c3),
                      _dptr(k3))
        return {"ind_freq": ind.astype(np.int64), "chijj3": c3, "chijj3_k": k3.reshape(N, nb)}

    def chijj(self):
        """Results of the last calc_chijj_vertex_corr_all_optim."""
        nk0, nw0, nbk, n8 = self.dims()
        NB = nw0 // 2 + 1
        c1, c2, kx0 = np.zeros(NB), np.zeros(NB), np.zeros(1)
        self.ctx.call("tpsc_get_chijj", _dptr(c1), _dptr(c2), _dptr(kx0), None, None)
        nb = getattr(self, "_nbins", 1)
        k1, k2 = np.zeros(NB * nb), np.zeros(NB * nb)
        self.ctx.call("tpsc_get_chijj", None, None, None, _dptr(k1), _dptr(k2))
        return {"chijj1": c1, "chijj2": c2, "kx0": float(kx0[0]), "chijj1_k": k1.reshape(NB, nb),
                "chijj2_k": k2.reshape(NB, nb)}

    def sigma_qn(self, nq=None):
        """sigma(iq_n) = (-kx0 - chi_jj(iq_n)) / q_n, n = 1..nq, with and without
        the vertex correction (the Kubo form; the reference stops at chi_jj and
        kx0).  Returns (sigma, sigma_bubble)."""
        nk0, nw0, nbk, n8 = self.dims()
        nq = nw0 // 2 if nq is None else int(nq)
        s, sb = np.zeros(nq), np.zeros(nq)
        self.ctx.call("tpsc_sigma_iqn", nq, _dptr(s), _dptr(sb))
        return s, sb

    def sigma_qn_sensitivities(self, nq=1, h=(1e-5, 1e-5, 1e-5)):
        """d sigma(iq_n)/d(U, mu, t') for n = 1..nq and dD/d(U, mu, t') by
        central differences of full FP64 device solves (steps h; mu a shift of
        mu0 at fixed n, t' at fixed n).  The context is solved again at its
        own parameters afterwards.  Returns (dsigma [3, nq], dD [3])."""
        steps = np.ascontiguousarray(np.asarray(h, dtype=np.float64).reshape(3))
        ds, dD = np.zeros((3, int(nq))), np.zeros(3)
        self.ctx.call("tpsc_sigma_iqn_fd", int(nq), _dptr(steps), _dptr(ds), _dptr(dD))
        self._nbins = 1
        return ds, dD

    def sigma_qn_vjp(self, cot):
        """The backward pair of sigma_qn: grad[p] = sum_n cot[n-1] d sigma(iq_n)
        / d theta_p, theta = (U, mu, t'), by one reverse pass on the device
        (mu a shift of mu0 at fixed n, t' at fixed n).  Needs a solve of the
        current grid.  Returns (grad [3], dD [3])."""
        c = np.ascontiguousarray(np.atleast_1d(np.asarray(cot, dtype=np.float64)))
        grad, dD = np.zeros(3), np.zeros(3)
        self.ctx.call("tpsc_sigma_iqn_bwd", int(c.size), _dptr(c), _dptr(grad), _dptr(dD))
        return grad, dD

    def sigma_pade(self, w, Nn=64, eta=0.0):
        """Pade continuation of sigma(iq_n), n = 1..Nn, to w + i eta:
        (sigma(w), sigma_bubble(w)) complex arrays."""
        w = np.ascontiguousarray(np.atleast_1d(np.asarray(w, dtype=np.float64)))
        out = np.zeros((2, w.size), dtype=np.complex128)
        self.ctx.call("tpsc_sigma_pade", int(Nn), _dptr(w), int(w.size), float(eta), _dptr(out.view(np.float64)))
        return out[0], out[1]


def pade_batch(x, y, z, ctx=None):
    """Batched continued-fraction Pade on the GPU: functions sampled at x[f, j]
    with values y[f, j], evaluated at the points z; returns [nf, len(z)]."""
    ctx = ctx or Context()
    x = np.ascontiguousarray(np.atleast_2d(np.asarray(x, dtype=np.complex128)))
    y = np.ascontiguousarray(np.atleast_2d(np.asarray(y, dtype=np.complex128)))
    z = np.ascontiguousarray(np.atleast_1d(np.asarray(z, dtype=np.complex128)))
    nf, Nn = y.shape
    x = np.ascontiguousarray(np.broadcast_to(x, (nf, Nn)))
    out = np.zeros((nf, z.size), dtype=np.complex128)
    ctx.call("tpsc_pade_batch", nf, Nn, _dptr(x.view(np.float64)), _dptr(y.view(np.float64)), int(z.size),
             _dptr(z.view(np.float64)), _dptr(out.view(np.float64)))
    return out


SCALAR_NAMES = None


def _scalar_names():
    global SCALAR_NAMES
    if SCALAR_NAMES is None:
        SCALAR_NAMES = list(_lib.SCALARS)
    return SCALAR_NAMES


def solve_points(params, ctx=None, streams=2):
    """tpsc_solve_points: the rows (nk0, Nw0, n, T, tp, tpp, t3, U) solved by
    shape groups in the Newton-form mixed solve, one graph launch per group.
    Returns (scalars [npts, TPSC_S_COUNT], status [npts], wall ms)."""
    ctx = ctx or Context()
    p = np.ascontiguousarray(params, dtype=np.float64)
    n = p.shape[0]
    res = np.zeros((n, len(_scalar_names())))
    st = np.zeros(n, dtype=np.int32)
    ms = np.zeros(1)
    ctx.call("tpsc_set_group_streams", int(streams))
    ctx.call("tpsc_solve_points", n, _dptr(p), _dptr(res), st.ctypes.data_as(_lib._ip), _dptr(ms))
    return res, st, float(ms[0])


def sweep_points(npts, seed=20261203):
    """The parameter-sweep workload (tpsc_sweep_points): npts rows
    (nk0, Nw0, n, T, tp, tpp, t3, U) from std::mt19937_64(seed)."""
    lib = _lib.load()
    out = np.zeros((npts, 8))
    rc = lib.tpsc_sweep_points(int(npts), C.c_ulonglong(seed), _dptr(out))
    if rc:
        raise _lib.TPSCError(rc, "tpsc_sweep_points")
    return out


class Batch:
    """Many independent solves (uneven lattices and cutoffs) on one GPU through
    the batched sweep (tpsc_batch_*): ``nstreams`` solver contexts, each fed by
    a host thread, points largest first."""

    def __init__(self, nstreams=4, device=0):
        self.lib = _lib.load()
        st = C.c_int(0)
        self.h = self.lib.tpsc_batch_create(int(device), int(nstreams), C.byref(st))
        if not self.h:
            raise _lib.TPSCError(st.value, "tpsc_batch_create")

    def _err(self, rc):
        raise _lib.TPSCError(rc, self.lib.tpsc_batch_last_error(self.h).decode())

    def solve(self, params, form=_lib.FORM_NEWTON | _lib.FORM_MIXED):
        """params: (npts, 8) rows (nk0, Nw0, n, T, tp, tpp, t3, U).  Returns
        (scalars [npts, TPSC_S_COUNT], status [npts], wall ms); a failing
        point has NaN scalars and its status, the others are solved."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        n = p.shape[0]
        res = np.zeros((n, len(_scalar_names())))
        st = np.zeros(n, dtype=np.int32)
        ms = C.c_double(0.0)
        self.lib.tpsc_batch_solve(self.h, int(form), n, _dptr(p), _dptr(res), st.ctypes.data_as(_lib._ip),
                                  C.byref(ms))
        return res, st, ms.value

    def tune(self, params, form=_lib.FORM_NEWTON | _lib.FORM_MIXED, max_streams=16):
        """Times the sample on 1, 2, 4, ... max_streams contexts and keeps the
        fastest count; returns {count: ms}."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        k = int(np.floor(np.log2(max_streams))) + 1
        ms = np.zeros(k)
        rc = self.lib.tpsc_batch_tune(self.h, int(form), p.shape[0], _dptr(p), int(max_streams), _dptr(ms))
        if rc:
            self._err(rc)
        return {2 ** i: float(ms[i]) for i in range(k)}

    CORR_COLUMNS = ("n", "T", "mu0", "vF", "Usp", "difRelsp", "Uch", "difRelch", "dblOcc", "xi_x", "xi_y",
                    "xiAs_x", "xiAs_y", "xi0_x", "xi0_y", "nbq", "qmax0", "qmax1", "chi0max")

    def corr_length(self, nk0, Nw0, params, dens, nD, Temp, nT, nsr=0.0, mu_fs=float("nan"),
                    form=_lib.FORM_REFERENCE):
        """chi::calc_corr_length (src/chi.cpp:931-981) on the solver contexts:
        rows [nD nT, 19] in CORR_COLUMNS order (density-major), per-point
        status and the wall time (ms).  params = (tp, tpp, t3, U); nsr > 0
        and mu_fs fix the sum rules' nsr and the Fermi surface's mu for every
        point, as the reference's own scan keeps its constructor's."""
        tp, tpp, t3, U = params
        d = np.ascontiguousarray(dens, dtype=np.float64)
        t = np.ascontiguousarray(Temp, dtype=np.float64)
        rows = np.zeros((nD * nT, len(self.CORR_COLUMNS)))
        st = np.zeros(nD * nT, dtype=np.int32)
        ms = C.c_double()
        rc = self.lib.tpsc_batch_corr_length(self.h, int(form), int(nk0), int(Nw0), tp, tpp, t3, U, _dptr(d),
                                             int(nD), _dptr(t), int(nT), float(nsr), float(mu_fs), _dptr(rows),
                                             st.ctypes.data_as(_lib._ip), C.byref(ms))
        if rc and not st.any():
            self._err(rc)
        return rows, st, ms.value

    def set_graph_mode(self, mode):
        """tpsc_set_graph_mode of every solver context (2: each Newton-form
        point is one graph launch, updated in place per point; 3: a Newton +
        mixed sweep by shape groups, one graph launch per (nk0, Nw0) group
        whose kernels each run over all its points)."""
        rc = self.lib.tpsc_batch_set_graph_mode(self.h, int(mode))
        if rc:
            self._err(rc)

    @property
    def nstreams(self):
        v = C.c_int(0)
        self.lib.tpsc_batch_streams(self.h, C.byref(v))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.tpsc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
