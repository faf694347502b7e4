"""The bounded grid barrier of the device root searches, made to run out.

k_sumrule_roots and k_mu_roots synchronise their cooperative grid with a
barrier whose spin is bounded (a second or two): a block that never arrives
must not hang the GPU.  tpsc_barrier_probe runs that barrier alone in a
cooperative launch of the same grid, with one block withheld: every other
block's wait runs out, sets the error flag and leaves, the kernel ends, and
the context is still usable for a solve.  Nothing faults and nothing hangs;
the withheld block simply returns without arriving.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _probe(g, withhold):
    err, out, blocks, ms = C.c_int(-1), C.c_int(-1), C.c_int(0), np.zeros(1)
    g.ctx.call("tpsc_barrier_probe", int(withhold), C.byref(err), C.byref(out), C.byref(blocks),
               ms.ctypes.data_as(C.POINTER(C.c_double)))
    return err.value, out.value, blocks.value, float(ms[0])


def test_barrier_passes_when_every_block_arrives_and_runs_out_when_one_does_not():
    from tpsc_conductivity_b200.api import Green

    g0 = load_golden("l16_w64_u2")
    p = g0["p"]
    g = Green(p["nk0"], p["Nw0"], p["n"], p["T"], 0.1, (p["tp"], p["tpp"], p["t3"], p["U"]))
    err, out, blocks, ms = _probe(g, -1)
    assert (err, out) == (0, 0)
    assert blocks >= 2
    err, out, blocks, ms = _probe(g, blocks - 1)
    print(f"withheld 1 of {blocks} blocks: error flag {err}, {out} blocks left with it after {ms:.0f} ms")
    assert err == 1
    assert out == blocks - 1       # every block that arrived gave up
    assert 100.0 < ms < 30000.0    # after its spin bound, not at once, not for long
    # the context is unharmed: a full solve still matches the reference
    g.solve()
    assert abs(g.scalars()["Usp"] - g0["s"]["Usp"]) <= 1e-9 * g0["s"]["Usp"]
