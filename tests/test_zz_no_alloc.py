"""The allocation-free sum rule (tpsc_sumrule_noalloc) against the context
entry point (tpsc_trace_diff_chi) on the same chi0.

tpsc_sumrule_noalloc exists for callers that cannot allocate device memory
where they need the sum rule (code inside a memory pool or arena, framework
callbacks that forbid allocation, solver loops that must not synchronise the
device through cudaMalloc/cudaFree).  Its partial sums live in a fixed device
array shared by all calls, so it is called twice in a row here: a second call
must not see the first call's leftovers.  This file is collected last so a
run that stops at the first failure has already run every other test.

The argument checks return before any device call, so they also run without
a GPU."""
import numpy as np
import pytest

from conftest import load_golden


# l256_w4096_u4 is the largest lattice the fixed array accepts: N8 = 8385
# octant points in 2097 of its 2100 partial-sum slots, the arrival counter
# right behind them
@pytest.mark.gpu
@pytest.mark.parametrize("name", ["l32_w256_u4_tp", "l64_w1024_u4", "l256_w4096_u4"])
def test_noalloc_sumrule_matches_context_entry_point(name):
    import torch

    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Green

    g = load_golden(name)
    p = g["p"]
    gr = Green(p["nk0"], p["Nw0"], p["n"], p["T"], 0.1, (p["tp"], p["tpp"], p["t3"], p["U"]))
    gr.calc_chiqw_FFT_spline()
    c = gr.chi0()
    dev = torch.device("cuda:0")
    chi = torch.from_numpy(np.ascontiguousarray(c["chiqw"])).to(dev)
    ci = torch.from_numpy(c["chi0_inf"]).to(dev)
    ci2 = torch.from_numpy(c["chi0_inf2"]).to(dev)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev).cuda_stream
    cases = [(0, 0.4 * g["s"]["Usp"]), (0, 0.9 * g["s"]["Usp"]), (1, 0.5 * p["U"]), (1, g["s"]["Uch"])]
    for call in range(2):
        for ch, Uv in cases:
            st = lib.tpsc_sumrule_noalloc(chi.data_ptr(), ci.data_ptr(), ci2.data_ptr(), p["nk0"], p["Nw0"],
                                          p["T"], ch, Uv, out.data_ptr(), stream)
            assert st == 0, (call, ch, Uv)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            t, dt = gr.traceDiffChi(ch, Uv)
            assert abs(got[0] - t) <= 1e-11 * abs(t), (call, ch, Uv, got[0], t)
            assert abs(got[1] - dt) <= 1e-11 * abs(dt), (call, ch, Uv, got[1], dt)
            out.fill_(float("nan"))


@pytest.mark.gpu
def test_noalloc_rejects_lattices_beyond_its_scratch():
    import torch

    from tpsc_conductivity_b200 import _lib

    lib = _lib.load()
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    p = dummy.data_ptr()
    assert lib.tpsc_sumrule_noalloc(p, p, p, 512, 64, 0.1, 0, 1.0, p, None) == 1  # TPSC_ERR_ARG


# (nk0, Nw0, T, channel): each violates one rule; the pointers are never read
BAD_ARGS = [
    (512, 64, 0.1, 0),   # beyond the fixed array (nk0 <= 256)
    (48, 64, 0.1, 0),    # nk0 not a power of two
    (4, 64, 0.1, 0),     # nk0 below 8
    (32, 63, 0.1, 0),    # odd Nw0
    (32, 2, 0.1, 0),     # Nw0 below 4
    (32, 64, 0.0, 0),    # T <= 0
    (32, 64, -0.1, 1),
    (32, 64, float("nan"), 1),
    (32, 64, 0.1, 2),    # channel neither 0 (spin) nor 1 (charge)
    (32, 64, 0.1, -1),
]


@pytest.mark.parametrize("nk0,Nw0,T,channel", BAD_ARGS)
def test_noalloc_rejects_bad_arguments_before_any_device_call(nk0, Nw0, T, channel):
    from tpsc_conductivity_b200 import _lib

    lib = _lib.load()
    fake = 256  # a non-null address that the argument checks never dereference
    assert lib.tpsc_sumrule_noalloc(fake, fake, fake, nk0, Nw0, T, channel, 1.0, fake, None) == 1  # TPSC_ERR_ARG


@pytest.mark.parametrize("which", range(4))
def test_noalloc_rejects_null_pointers(which):
    from tpsc_conductivity_b200 import _lib

    lib = _lib.load()
    ptrs = [256, 256, 256, 256]
    ptrs[which] = None
    chi, ci, ci2, out = ptrs
    assert lib.tpsc_sumrule_noalloc(chi, ci, ci2, 32, 64, 0.1, 0, 1.0, out, None) == 1
