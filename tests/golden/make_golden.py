"""Regenerate the golden fixtures in this folder from the reference itself.

Runs ``oracle/_ref/tpsc_ref_probe`` -- the UNMODIFIED reference sources
compiled by ``oracle/ref/Makefile`` (``TPSC_REFERENCE_SRC=<checkout>/src make -C
oracle/ref``) -- on a set of
small lattices and stores what it computed as ``<name>.npz``.  Needs the
reference checkout to build the probe; the fixtures themselves travel with the
repository and are all the tests read.

usage: python tests/golden/make_golden.py [--threads 8] [--only name ...]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PROBE = os.path.join(ROOT, "oracle", "_ref", "tpsc_ref_probe")

# name: (mode, U, tp, tpp, t3, n, T, nk0, Nw0, keep_full_arrays[, angle bins of chi_jj[, mmin]])
CASES = {
    # tiny lattice, half-grid pre-pass exercised, conductivity too
    "l16_w64_u2": ("cond", 2.0, 0.0, 0.0, 0.0, 0.875, 0.25, 16, 64, True),
    # the 32x32 plain-TPSC case: t'=0, U=2, n=0.875, T=0.25, 256 positive iwn
    "l32_w512_u2": ("cond", 2.0, 0.0, 0.0, 0.0, 0.875, 0.25, 32, 512, True),
    # next-nearest and third-neighbour hoppings
    "l32_w256_u4_tp": ("cond", 4.0, -0.15, 0.05, 0.02, 0.875, 0.1, 32, 256, True),
    # electron doping n > 1 (nsr = 2 - n branch, src/chi.cpp:18, 370)
    "l16_w128_n110": ("cond", 3.0, -0.2, 0.1, 0.0, 1.1, 0.2, 16, 128, True),
    # half filling, particle-hole symmetric: mu0 = 0 shortcut (src/green0.cpp:18-23)
    "l16_w64_half": ("cond", 2.0, 0.0, 0.0, 0.0, 1.0, 0.3, 16, 64, True),
    # chi_jj resolved into 3 angle bins (N_theta_k)
    "l32_w256_theta3": ("cond", 3.0, -0.1, 0.0, 0.0, 0.9, 0.1, 32, 256, True, 3),
    # the optical-conductivity case: 128x128, U=3, n=0.9, T=0.1, 1024 positive
    # fermionic frequencies; scalars, sampled columns, chi_jj and 4 angle bins
    "l128_w2048_cond": ("cond", 3.0, 0.0, 0.0, 0.0, 0.9, 0.1, 128, 2048, False, 4),
    # chi_jj (bubble + Maki-Thompson, kx0) at 256x256 with 2048 positive iwn
    "l256_w4096_cond": ("cond", 4.0, -0.15, 0.0, 0.0, 0.875, 0.05, 256, 4096, False),
    # the Aslamazov-Larkin correction chijj3 on the non-uniform iqn grid of
    # mmin (src/cond_opt.cpp:4292-6529), with the reference's chijj3_qn_*,
    # chijj_with_all_vc_qn_* and (angle bins) chijj3_k_qn_* files
    "al_l16_w64": ("cond3", 2.0, -0.1, 0.0, 0.0, 0.875, 0.25, 16, 64, True, 1, 3),
    "al_l32_w256_theta3": ("cond3", 4.0, -0.15, 0.0, 0.0, 0.875, 0.2, 32, 256, True, 3, 3),
    "al_l16_w128_n110": ("cond3", 2.5, -0.2, 0.05, 0.0, 1.1, 0.3, 16, 128, True, 1, 2),
    "al_l32_w512_n1": ("cond3", 3.0, -0.1, 0.0, 0.0, 1.0, 0.15, 32, 512, True, 1, 4),
    # larger lattice, lower temperature
    "l64_w1024_u4": ("solve", 4.0, -0.15, 0.0, 0.0, 0.875, 0.05, 64, 1024, False),
    # the 256x256, 2048 positive iwn case: scalars and sampled columns only
    "l256_w4096_u4": ("solve", 4.0, -0.15, 0.0, 0.0, 0.875, 0.05, 256, 4096, False),
    # the saved-run files (chi0 binary, self_bin, self_tpsc ascii, Green ascii)
    # as the reference's own writers leave them, byte for byte, on a 16x16
    # lattice with 16 positive iwn
    "files_l16_w32": ("files", 2.0, -0.1, 0.0, 0.0, 0.875, 0.25, 16, 32, True),
    # chi::calc_corr_length over n in {0.85, 0.9}, T in {0.2, 0.3} on a 16x16
    # lattice with 32 positive iwn: the reference's corrLgth file
    "corr_l16_w64": ("corr", 2.5, -0.1, 0.0, 0.0, 0.85, 0.2, 16, 64, True),
    # green::calc_Self_Re_w_BZ on a 16x16 lattice with 32 positive iwn: the
    # Pade and J-fraction Sigma(k, w + i eta) and A(k, w) files of every k
    "rew_l16_w64": ("rew", 3.0, -0.15, 0.0, 0.0, 0.9, 0.15, 16, 64, True),
    # green::EDC, both overloads, on a 16x16 lattice with 16 positive iwn
    "edc_l16_w32": ("edc", 2.5, -0.1, 0.0, 0.0, 0.9, 0.25, 16, 32, True),
    # the infinite lattice: chi0::calc_chi0_qlims at n = 0, 1 (adaptive
    # quadrature), the infinite-system mu0, chiqw_discret on the 16x16 lattice
    "chi0inf_l16": ("chi0inf", 2.0, -0.15, 0.05, 0.0, 0.85, 0.2, 16, 32, True),
}

# the files the reference's writers leave (src/chi0.cpp:63, src/green.cpp:1507,
# 1557, 1606); chi0_qmax_wn_* and chi0_wn0_q_* are the chi0 stage's own dumps
FILE_PREFIXES = ("chi0_", "self_bin_", "self_tpsc_", "Green_", "corrLgth_", "Self_Re_w_", "spectr_wgt_", "edc")
FILE_SKIP = ("chi0_qmax_wn_", "chi0_wn0_q_")


def read_meta(path):
    meta = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2:
                meta[parts[0]] = parts[1]
    return meta


def run_case(name, spec, threads):
    mode, U, tp, tpp, t3, n, T, nk0, Nw0, full = spec[:10]
    ntheta = spec[10] if len(spec) > 10 else 1
    mmin = spec[11] if len(spec) > 11 else 3
    with tempfile.TemporaryDirectory() as d:
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), TPSC_PROBE_NTHETA=str(ntheta),
                   TPSC_PROBE_MMIN=str(mmin))
        args = [PROBE, d, mode] + [repr(v) for v in (U, tp, tpp, t3, n, T)] + [str(nk0), str(Nw0)]
        subprocess.run(args, check=True, env=env)
        meta = read_meta(os.path.join(d, "meta.txt"))
        nbk = nk0 // 2 + 1
        if mode == "chi0inf":
            work = os.path.join(d, "work")
            names = sorted(f for f in os.listdir(work) if f.startswith("chi0_q_"))
            out = {"params": np.array([U, tp, tpp, t3, n, T, nk0, Nw0], dtype=np.float64),
                   "mu0_inf": np.array(float(meta["mu0_inf"])), "mu0_finite": np.array(float(meta["mu0_finite"])),
                   "chi_discret": np.array(float(meta["chi_discret"])), "file_names": np.array(names)}
            for i, f in enumerate(names):
                out[f"file_{i}"] = np.fromfile(os.path.join(work, f), dtype=np.uint8)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
            print(name, "done", names, meta.get("t_chi0inf"))
            return
        if mode == "corr":
            work = os.path.join(d, "work")
            names = sorted(f for f in os.listdir(work) if f.startswith("corrLgth_"))
            out = {"params": np.array([U, tp, tpp, t3, n, T, nk0, Nw0], dtype=np.float64),
                   "dens": np.array([n, n + 0.05]), "temp": np.array([T, 1.5 * T]),
                   "file_names": np.array(names)}
            for i, f in enumerate(names):
                out[f"file_{i}"] = np.fromfile(os.path.join(work, f), dtype=np.uint8)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
            print(name, "done", names)
            return
        n8 = nbk * (nbk + 1) // 2
        nw = Nw0 // 2 + 1

        def rd(fname, shape=None, cplx=False):
            a = np.fromfile(os.path.join(d, fname), dtype=np.float64)
            if cplx:
                a = a[0::2] + 1j * a[1::2]
            return a.reshape(shape) if shape else a

        out = {
            "params": np.array([U, tp, tpp, t3, n, T, nk0, Nw0], dtype=np.float64),
            "scalars_names": np.array(["mu0", "chi0max", "qmax0", "qmax1", "Usp", "Uch", "dblOcc",
                                       "Sigma_inf", "mu"]),
            "scalars": np.array([float(meta[k]) for k in ["mu0", "chi0max", "qmax0", "qmax1", "Usp",
                                                         "Uch", "dblOcc", "Sigma_inf", "mu"]]),
            "chi0_inf": rd("chi0_inf.bin"),
            "chi0_inf2": rd("chi0_inf2.bin"),
            "dtau_chirt0": rd("dtau_chirt0.bin"),
            "sigma_inf2": rd("sigma_inf2.bin"),
            "sigma_inf3": rd("sigma_inf3.bin"),
            "sigma_inf4": rd("sigma_inf4.bin"),
            "ref_seconds": np.array([float(meta.get(k, 0.0)) for k in
                                     ["t_self", "t_traceSelfG", "t_find_mu"]]),
            "ref_threads": np.array(int(meta["omp_threads"])),
            # chi::sp_corr_length (src/chi.cpp:450-718) after the solve
            "corr_names": np.array(["vF", "xi_y", "xi_x", "xiAs_y", "xiAs_x", "xi0_y", "xi0_x"]),
            "corr": np.array([float(meta[k]) for k in ["vF", "xi_y", "xi_x", "xiAs_y", "xiAs_x", "xi0_y", "xi0_x"]]),
        }
        chiqw = rd("chiqw.bin", (nw, n8))
        V = rd("vertex_rt.bin", (nw, n8))
        S = rd("self.bin", (Nw0 // 2, n8), cplx=True)
        if full:
            out["chiqw"] = chiqw
            out["vertex_rt"] = V
            out["self"] = S
        else:
            cols = np.unique(np.linspace(0, n8 - 1, 12).astype(np.int64))
            out["cols"] = cols
            out["chiqw_cols"] = chiqw[:, cols]
            out["vertex_rt_cols"] = V[:, cols]
            out["self_cols"] = S[:, cols]
            out["chiqw_w0"] = chiqw[0]
        if mode in ("cond", "cond3"):
            out["kx0"] = np.array(float(meta["kx0"]))
            out["chijj1"] = rd("chijj1.bin")
            out["chijj2"] = rd("chijj2.bin")
            # text outputs of find_FS_inter, MDC (10 points, w = 0, 4 etas) and
            # Gwn_local as the reference writes them (src/green.cpp:2227-2330,
            # 1020-1060, 226-263); the probe runs them as tpsc_main.cpp does
            work = os.path.join(d, "work")

            def table(prefix, exclude=None):
                f = [x for x in os.listdir(work)
                     if x.startswith(prefix) and not (exclude and x.startswith(exclude))]
                return np.loadtxt(os.path.join(work, f[0]), ndmin=2)

            if ntheta > 1:
                # chijj1_k_qn_* / chijj2_k_qn_*: lines "j  p+1  value" (src/cond_opt.cpp:3931-3941)
                for key, prefix in (("chijj1_k", "chijj1_k_qn_"), ("chijj2_k", "chijj2_k_qn_")):
                    t = table(prefix)
                    out[key] = t[:, 2].reshape(nw, ntheta)
            out["mdc_A"] = table("Akw_Pade_k_")[:, 2:]
            sp = table("Self_Pade_k_")[:, 2:]
            out["mdc_sigma"] = sp[:, 0::2] + 1j * sp[:, 1::2]
            g = table("Gwn_loc_")
            out["gwn_local"] = g[:, 1] + 1j * g[:, 2]
            out["fs_inter"] = table("FS_inter_AkF_", exclude="FS_inter_AkF_Pade_")
            out["fs_inter_pade"] = table("FS_inter_AkF_Pade_")
        if mode == "cond3":
            work = os.path.join(d, "work")
            out["mmin"] = np.array(mmin)
            out["chijj3"] = rd("chijj3.bin")
            names = sorted(f for f in os.listdir(work)
                           if f.startswith(("chijj3_qn_", "chijj_with_all_vc_qn_", "chijj3_k_qn_", "chijj3_k_tot_qn_")))
            out["file_names"] = np.array(names)
            for i, f in enumerate(names):
                out[f"file_{i}"] = np.fromfile(os.path.join(work, f), dtype=np.uint8)
            t = np.loadtxt(os.path.join(work, [f for f in names if f.startswith("chijj3_qn_")][0]), ndmin=2)
            out["ind_freq"] = t[:, 0].astype(np.int64)
            if ntheta > 1:
                t = np.loadtxt(os.path.join(work, [f for f in names if f.startswith("chijj3_k_qn_")][0]), ndmin=2)
                out["chijj3_k"] = t[:, 2].reshape(-1, ntheta)
        if mode in ("files", "rew", "edc"):
            work = os.path.join(d, "work")
            names = sorted(f for f in os.listdir(work)
                           if f.startswith(FILE_PREFIXES) and not f.startswith(FILE_SKIP))
            out["file_names"] = np.array(names)
            for i, f in enumerate(names):
                out[f"file_{i}"] = np.fromfile(os.path.join(work, f), dtype=np.uint8)
            out["ek"] = rd("ek.bin", (nbk, nbk))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "done", {k: meta.get(k) for k in ("Usp", "Uch", "mu")})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--only", nargs="*")
    a = ap.parse_args()
    if not os.path.exists(PROBE):
        raise SystemExit("build the reference probe first: TPSC_REFERENCE_SRC=<reference>/src make -C oracle/ref")
    for name, spec in CASES.items():
        if a.only and name not in a.only:
            continue
        run_case(name, spec, a.threads)


if __name__ == "__main__":
    main()
