"""ctypes binding of the C ABI in include/tpsc_b200.h.

The shared library is the in-tree ``libtpsc_b200.so`` built by
``tpsc_conductivity_b200.build``.  There is no fallback: if the library is
missing or no CUDA device is present, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libtpsc_b200.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

# (name, restype, argtypes) -- the exact exports of include/tpsc_b200.h
SIGNATURES = [
    ("tpsc_create", C.c_void_p, [C.c_int, _ip]),
    ("tpsc_destroy", None, [C.c_void_p]),
    ("tpsc_last_error", C.c_char_p, [C.c_void_p]),
    ("tpsc_set_model", C.c_int, [C.c_void_p, C.c_int, C.c_int] + [C.c_double] * 6),
    ("tpsc_chi0", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("tpsc_trace_chi0", C.c_int, [C.c_void_p, _dp]),
    ("tpsc_trace_diff_chi", C.c_int, [C.c_void_p, C.c_int, C.c_double, _dp, _dp]),
    ("tpsc_find_Usp_Uch_grid", C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp]),
    ("tpsc_find_Usp_Uch", C.c_int, [C.c_void_p]),
    ("tpsc_sp_corr_length", C.c_int, [C.c_void_p, _dp]),
    ("tpsc_sp_corr_length_fs", C.c_int, [C.c_void_p, C.c_double, _dp]),
    ("tpsc_sumrule_tangents", C.c_int, [C.c_void_p, _dp]),
    ("tpsc_get_self_async", C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    ("tpsc_get_sigma32_async", C.c_int, [C.c_void_p, C.c_void_p]),
    ("tpsc_set_self", C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    ("tpsc_set_chi0", C.c_int, [C.c_void_p, _dp]),
    ("tpsc_get_sigma_tau", C.c_int, [C.c_void_p, C.c_int, _dp]),
    ("tpsc_mu0_infinite", C.c_int, [C.c_void_p, _dp, _ip]),
    ("tpsc_chi0_infinite", C.c_int, [C.c_void_p, C.c_double, C.c_int, _dp, C.c_int, _dp, _ip]),
    ("tpsc_file_name", C.c_int, [C.c_int, C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("tpsc_write_chi0_bin", C.c_int, [C.c_char_p, C.c_int, C.c_int, _dp]),
    ("tpsc_read_chi0_bin", C.c_int, [C.c_char_p, _ip, _ip, _dp, C.c_longlong]),
    ("tpsc_write_self_bin", C.c_int, [C.c_char_p, C.c_int, C.c_int, _dp, _dp]),
    ("tpsc_read_self_bin", C.c_int, [C.c_char_p, C.c_int, C.c_int, _dp]),
    ("tpsc_write_self_ascii", C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _dp]),
    ("tpsc_read_self_ascii", C.c_int, [C.c_char_p, C.c_int, C.c_int, _dp]),
    ("tpsc_write_green_ascii", C.c_int, [C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.c_double, _dp, C.c_longlong]),
    ("tpsc_wait_copies", C.c_int, [C.c_void_p, C.c_int]),
    ("tpsc_sumrule_vjp", C.c_int, [C.c_void_p, _dp, _dp]),
    ("tpsc_set_mu_shift", C.c_int, [C.c_void_p, C.c_double]),
    ("tpsc_batch_create", C.c_void_p, [C.c_int, C.c_int, _ip]),
    ("tpsc_batch_destroy", None, [C.c_void_p]),
    ("tpsc_batch_last_error", C.c_char_p, [C.c_void_p]),
    ("tpsc_batch_streams", C.c_int, [C.c_void_p, _ip]),
    ("tpsc_batch_set_graph_mode", C.c_int, [C.c_void_p, C.c_int]),
    ("tpsc_batch_corr_length", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_double, _dp, C.c_int, _dp, C.c_int, C.c_double, C.c_double, _dp, _ip,
                                         _dp]),
    ("tpsc_batch_solve", C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _ip, _dp]),
    ("tpsc_batch_tune", C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _dp]),
    ("tpsc_sweep_points", C.c_int, [C.c_int, C.c_ulonglong, _dp]),
    ("tpsc_vertex", C.c_int, [C.c_void_p]),
    ("tpsc_self_energy", C.c_int, [C.c_void_p]),
    ("tpsc_trace_self_G", C.c_int, [C.c_void_p, _dp]),
    ("tpsc_trace_diff_G", C.c_int, [C.c_void_p, C.c_double, _dp, _dp]),
    ("tpsc_find_mu", C.c_int, [C.c_void_p]),
    ("tpsc_solve", C.c_int, [C.c_void_p]),
    ("tpsc_get_scalars", C.c_int, [C.c_void_p, _dp, C.c_int]),
    ("tpsc_get_dims", C.c_int, [C.c_void_p, _ip]),
    ("tpsc_get_ek", C.c_int, [C.c_void_p, _dp]),
    ("tpsc_get_chi0", C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    ("tpsc_get_vertex", C.c_int, [C.c_void_p, _dp]),
    ("tpsc_get_self", C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    ("tpsc_stage_times", C.c_int, [C.c_void_p, _dp, C.c_int]),
    ("tpsc_get_stream", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("tpsc_run_kernel", C.c_int, [C.c_void_p, C.c_int]),
    ("tpsc_kernel_bytes", C.c_int, [C.c_void_p, C.c_int, _dp]),
    ("tpsc_launch_count", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    ("tpsc_fma_peak", C.c_int, [C.c_int, _dp]),
    ("tpsc_pade_sigma", C.c_int, [C.c_void_p, _ip, C.c_int, _dp, C.c_int, C.c_int, _dp, _dp]),
    ("tpsc_gwn_local", C.c_int, [C.c_void_p, _dp]),
    ("tpsc_set_form", C.c_int, [C.c_void_p, C.c_int]),
    ("tpsc_set_graph_mode", C.c_int, [C.c_void_p, C.c_int]),
    ("tpsc_set_nsr", C.c_int, [C.c_void_p, C.c_double]),
    ("tpsc_tune_tau_tiles", C.c_int, [C.c_void_p, C.c_int, _dp]),
    ("tpsc_tune_tau_plans", C.c_int, [C.c_void_p, C.c_int, _dp]),
    ("tpsc_set_tau_tile", C.c_int, [C.c_int, C.c_int, C.c_int]),
    ("tpsc_set_slice_plan", C.c_int, [C.c_int, C.c_int, C.c_int]),
    ("tpsc_get_slice_plan", C.c_int, [C.c_int, C.c_int]),
    ("tpsc_tensor_plan_errors", C.c_int, [C.c_void_p, C.c_int]),
    ("tpsc_tune_slice_plans", C.c_int, [C.c_void_p, C.c_int, _dp]),
    ("tpsc_graph_stats", C.c_int, [C.c_void_p, C.c_void_p]),
    ("tpsc_chijj", C.c_int, [C.c_void_p, C.c_int]),
    ("tpsc_get_chijj", C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    ("tpsc_chijj3", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("tpsc_barrier_probe", C.c_int, [C.c_void_p, C.c_int, _ip, _ip, _ip, _dp]),
    ("tpsc_get_chijj3", C.c_int, [C.c_void_p, C.c_int, _ip, _ip, _dp, _dp]),
    ("tpsc_sigma_iqn", C.c_int, [C.c_void_p, C.c_int, _dp, _dp]),
    ("tpsc_sigma_iqn_fd", C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp]),
    ("tpsc_sigma_iqn_bwd", C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp]),
    ("tpsc_solve_points", C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _ip, _dp]),
    ("tpsc_set_group_streams", C.c_int, [C.c_void_p, C.c_int]),
    ("tpsc_sigma_pade", C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int, C.c_double, _dp]),
    ("tpsc_pade_batch", C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _dp]),
    ("tpsc_sumrule_noalloc", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, C.c_void_p,
      C.c_void_p]),
]

# enum tpsc_form (flags)
FORM_REFERENCE, FORM_NEWTON, FORM_MIXED = 0, 1, 2
# enum tpsc_file_kind
FILE_CHI0_BIN, FILE_SELF_BIN, FILE_SELF_ASCII, FILE_GREEN = 0, 1, 2, 3

# tpsc_run_kernel stage ids
KERNELS = ["gslice", "chi0_slice", "chi0_tau", "vertex_q", "vertex_tau", "sigma_slice", "sigma_tau",
           "sumrule", "trace_diff_G", "chi0_slice+tau", "sumrule_newton", "trace_diff_G_newton",
           "sumrule_moments", "sumrule_roots", "sigma_moments", "sigma_moments+mu_roots"]

STATUS = {0: "OK", 1: "bad argument", 2: "CUDA error", 3: "out of device memory",
          4: "root not found", 5: "stage prerequisite missing", 6: "non-finite result"}
OK, ERR_ARG, ERR_CUDA, ERR_OOM, ERR_NO_ROOT, ERR_STATE, ERR_NONFINITE = range(7)

# enum tpsc_scalar
SCALARS = ["mu0", "chi0max", "qmax0", "qmax1", "Usp", "Uch", "dblOcc", "difRelsp", "difRelch",
           "Sigma_inf", "mu", "trSG", "trSG_asymp", "trSG2", "dblOcc_SG2", "trChi0", "trChi0_corr",
           "evals_sp", "evals_ch", "evals_mu"]


class TPSCError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Load (once) the CUDA library; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build it with `python -m tpsc_conductivity_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(p)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(lib, ctx, status: int):
    if status != 0:
        msg = lib.tpsc_last_error(ctx)
        raise TPSCError(status, msg.decode() if msg else "")
