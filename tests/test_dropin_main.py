"""The reference's own driver (src/tpsc_main.cpp, compiled unchanged against
the drop-in classes of tpsc_conductivity_b200/dropin) runs on the GPU from an
input.dat and writes the reference's result files with the reference's
numbers."""
import glob
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden

BIN = os.path.join(ROOT, "tpsc_conductivity_b200", "dropin", "_build", "tpsc_main_b200")


def read_params(path):
    out = {}
    for line in open(path):
        f = line.split()
        if len(f) >= 2:
            out[f[0].rstrip(":")] = float(f[1])
    return out


@pytest.mark.gpu
def test_reference_main_runs_on_the_dropin(tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("tpsc_main_b200 is built only where the reference checkout exists (make -C .../dropin)")
    g = load_golden("l32_w512_u2")
    p, s = g["p"], g["s"]
    run = tmp_path / "a" / "b"
    run.mkdir(parents=True)
    # U tp tpp t3 n T nk0 Nw0 chijj3 mmin (src/tpsc_main.cpp:33)
    (tmp_path / "input.dat").write_text(
        f"{p['U']} {p['tp']} {p['tpp']} {p['t3']} {p['n']} {p['T']} {p['nk0']} {p['Nw0']} 0 3\n")
    r = subprocess.run([BIN], cwd=run, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    params = read_params(glob.glob(str(run / "TPSCparams_*"))[0])
    for k in ("Usp", "Uch", "mu", "mu0"):
        assert abs(params[k] - s[k]) <= 1e-9 * max(1.0, abs(s[k])), (k, params[k], s[k])
    infos = open(glob.glob(str(run / "TPSC_infos_*"))[0]).read()
    assert "double occupation (Self*G2)" in infos
    gl = np.loadtxt(glob.glob(str(run / "Gwn_loc_*"))[0])
    assert np.allclose(gl[:, 1] + 1j * gl[:, 2], g["gwn_local"], rtol=1e-8, atol=1e-10)
    A = np.loadtxt(glob.glob(str(run / "Akw_Pade_k_*"))[0])
    assert np.allclose(A[:, 2:], g["mdc_A"], rtol=1e-6, atol=1e-11)
    fs = np.loadtxt(glob.glob(str(run / "FS_inter_AkF_Pade_*"))[0])
    assert np.allclose(fs[:, 2], g["fs_inter_pade"][:, 2], rtol=1e-6)


COND_BIN = os.path.join(ROOT, "tpsc_conductivity_b200", "dropin", "_build", "cond_main_b200")


@pytest.mark.gpu
def test_conductivity_block_writes_the_reference_files(tmp_path):
    """The conductivity block of src/tpsc_main.cpp (cond_opt +
    calc_chijj_vertex_corr_all_optim) on the drop-in classes writes
    chijj1_qn_*, chijj2_qn_*, chijj_with_vc1_qn_*, kx0_*, kx0_bin_* and the
    angle-resolved chijj*_k_qn_* / chijj*_k_tot_qn_* with the reference's
    numbers."""
    if not os.path.exists(COND_BIN):
        pytest.skip("cond_main_b200 is built by make -C tpsc_conductivity_b200/dropin")
    g = load_golden("l32_w256_theta3")
    p = g["p"]
    nt = g["chijj1_k"].shape[1]
    run = tmp_path / "a" / "b"
    run.mkdir(parents=True)
    (tmp_path / "input.dat").write_text(
        f"{p['U']} {p['tp']} {p['tpp']} {p['t3']} {p['n']} {p['T']} {p['nk0']} {p['Nw0']} 0 3 {nt}\n")
    r = subprocess.run([COND_BIN], cwd=run, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "difference relative avec -k0" in r.stdout

    def one(prefix):
        return glob.glob(str(run / prefix))[0]

    s1, s2 = np.max(np.abs(g["chijj1"])), np.max(np.abs(g["chijj2"]))
    c1 = np.loadtxt(one("chijj1_qn_*"))
    c2 = np.loadtxt(one("chijj2_qn_*"))
    cv = np.loadtxt(one("chijj_with_vc1_qn_*"))
    assert np.array_equal(c1[:, 0], np.arange(p["Nw0"] // 2 + 1))
    assert np.max(np.abs(c1[:, 1] - g["chijj1"])) <= 1e-10 * s1
    assert np.max(np.abs(c2[:, 1] - g["chijj2"])) <= 1e-10 * s2
    assert np.max(np.abs(cv[:, 1] - (g["chijj1"] + g["chijj2"]))) <= 1e-10 * s1
    kx0 = float(open(one("kx0_[0-9]*")).read())
    assert abs(kx0 - float(g["kx0"])) <= 1e-10 * abs(float(g["kx0"]))
    kb = np.fromfile(one("kx0_bin_*"), dtype=np.float64)
    assert kb.size == 1 and kb[0] == kx0
    k1 = np.loadtxt(one("chijj1_k_qn_*"))
    k2 = np.loadtxt(one("chijj2_k_qn_*"))
    assert np.array_equal(k1[:nt, 1], np.arange(1, nt + 1))
    assert np.max(np.abs(k1[:, 2].reshape(-1, nt) - g["chijj1_k"])) <= 1e-10 * s1
    assert np.max(np.abs(k2[:, 2].reshape(-1, nt) - g["chijj2_k"])) <= 1e-10 * s2
    t1 = np.loadtxt(one("chijj1_k_tot_qn_*"))
    assert np.allclose(t1[:, 1], t1[:, 2], rtol=1e-12, atol=0)
    # the Fermi-surface files of find_FS_inter come first, as in the reference
    assert glob.glob(str(run / "FS_inter_AkF_Pade_*"))


@pytest.mark.gpu
def test_conductivity_block_with_the_al_correction_writes_its_files(tmp_path):
    """The same block with chijj3 = 1 in input.dat: the Aslamazov-Larkin
    correction on the non-uniform grid of mmin, and the reference's
    chijj3_qn_*, chijj_with_all_vc_qn_*, chijj3_k_qn_* and chijj3_k_tot_qn_*
    files (src/cond_opt.cpp:6448-6521) with the reference's grid and numbers."""
    import io

    if not os.path.exists(COND_BIN):
        pytest.skip("cond_main_b200 is built by make -C tpsc_conductivity_b200/dropin")
    g = load_golden("al_l32_w256_theta3")
    p = g["p"]
    nt = g["chijj3_k"].shape[1]
    mmin = int(g["mmin"])
    run = tmp_path / "a" / "b"
    run.mkdir(parents=True)
    (tmp_path / "input.dat").write_text(
        f"{p['U']} {p['tp']} {p['tpp']} {p['t3']} {p['n']} {p['T']} {p['nk0']} {p['Nw0']} 1 {mmin} {nt}\n")
    r = subprocess.run([COND_BIN], cwd=run, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "calcul de la seconde correction de vertex" in r.stdout
    names = [str(n) for n in g["file_names"]]
    scale = np.max(np.abs(g["chijj3"]))
    for prefix in ("chijj3_qn_", "chijj_with_all_vc_qn_", "chijj3_k_qn_", "chijj3_k_tot_qn_"):
        i = [k for k, n in enumerate(names) if n.startswith(prefix)]
        assert len(i) == 1, prefix
        ref_name = names[i[0]]
        mine = run / ref_name
        assert mine.exists(), ref_name  # same file name (parameters, nk0, Nw0, mmin)
        a = np.loadtxt(mine, ndmin=2)
        b = np.loadtxt(io.BytesIO(g[f"file_{i[0]}"].tobytes()), ndmin=2)
        assert a.shape == b.shape, prefix
        assert np.array_equal(a[:, 0], b[:, 0]), prefix  # the grid indices
        if prefix == "chijj3_k_tot_qn_":
            # total of the bins, total, their ratio
            assert np.max(np.abs(a[:, 1:3] - b[:, 1:3])) <= 1e-10 * scale
            assert np.allclose(a[:, 3], b[:, 3], rtol=1e-8, atol=0)
        elif prefix == "chijj3_k_qn_":
            assert np.array_equal(a[:, 1], b[:, 1])
            assert np.max(np.abs(a[:, 2] - b[:, 2])) <= 1e-10 * scale
        else:
            s = np.max(np.abs(b[:, 1]))
            assert np.max(np.abs(a[:, 1] - b[:, 1])) <= 1e-10 * s, prefix
