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
