import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: CPU test that takes more than a few seconds")


GOLDEN = os.path.join(ROOT, "tests", "golden")


def load_golden(name):
    import numpy as np

    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    names = [str(s) for s in d.get("scalars_names", [])]
    d["s"] = dict(zip(names, d["scalars"].tolist())) if names else {}
    U, tp, tpp, t3, n, T, nk0, Nw0 = d["params"].tolist()
    d["p"] = dict(U=U, tp=tp, tpp=tpp, t3=t3, n=n, T=T, nk0=int(nk0), Nw0=int(Nw0))
    return d


def golden_names():
    """The solve fixtures (scalars and arrays of a reference solve); the scan
    fixtures (corr_*) hold only the files the reference wrote."""
    import numpy as np

    out = []
    for f in sorted(os.listdir(GOLDEN)):
        if f.endswith(".npz") and "scalars_names" in np.load(os.path.join(GOLDEN, f)).files:
            out.append(f[:-4])
    return out


@pytest.fixture
def golden():
    return load_golden
