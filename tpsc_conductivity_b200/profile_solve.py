"""Repeated TPSC solves of one model, for profilers and stage timing.

    python -m tpsc_conductivity_b200.profile_solve --nk0 256 --nw0 4096 --form mixed_newton --solves 3

The model defaults to the bench's workload (t' = -0.15, t'' = t''' = 0,
U = 4, n = 0.875, T = 0.05) on the lattice and Matsubara grid given.  Every solve
is a full tpsc_solve on the library's stream; the last one's stage times
(ms, CUDA events) and root-search evaluation counts are printed as one JSON
line.  Under a kernel profiler, the launches of the last solve start at its
k_gk_table launch.  With --cond, every solve is followed by the
current-current correlator (bubble + Maki-Thompson, N_theta_k = 1), whose
stage times are in the same line.  --model takes the lattice parameters
"tp,U,n,T" (default the bench's -0.15,4,0.875,0.05).  --slice-plans sets the
plan of the four FP32 slice transforms (G, chi0, V, Sigma) for this lattice
before the first solve, e.g. 0,0,0,2 for the tensor-core Sigma slice.
"""
import argparse
import json

from . import _lib
from .api import CondOpt

FORMS = {
    "fp64_reference_roots": _lib.FORM_REFERENCE,
    "fp64_newton": _lib.FORM_NEWTON,
    "mixed_newton": _lib.FORM_NEWTON | _lib.FORM_MIXED,
}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--nk0", type=int, default=256)
    ap.add_argument("--nw0", type=int, default=4096)
    ap.add_argument("--form", choices=sorted(FORMS), default="mixed_newton")
    ap.add_argument("--solves", type=int, default=3)
    ap.add_argument("--cond", action="store_true")
    ap.add_argument("--model", default="-0.15,4,0.875,0.05")
    ap.add_argument("--slice-plans", default=None, help="plans of the G, chi0, V and Sigma slices, e.g. 0,0,0,2")
    a = ap.parse_args(argv)
    if a.slice_plans:
        lib = _lib.load()
        for kind, plan in enumerate(int(x) for x in a.slice_plans.split(",")):
            if lib.tpsc_set_slice_plan(kind, a.nk0, plan) != 0:
                raise SystemExit(f"slice plan {plan} is not available for kind {kind} at nk0 = {a.nk0}")
    tp, U, n, T = (float(x) for x in a.model.split(","))
    g = CondOpt(a.nk0, a.nw0, n, T, 0.1, (tp, 0.0, 0.0, U))
    g.set_form(FORMS[a.form])
    for _ in range(a.solves):
        g.solve()
        if a.cond:
            g.calc_chijj_vertex_corr_all_optim(False, 3, 1)
    s = g.scalars()
    print(json.dumps({"nk0": a.nk0, "nw0": a.nw0, "form": a.form, "slice_plans": a.slice_plans,
                      "stage_ms": g.stage_times(),
                      "evals": {"sp": s["evals_sp"], "ch": s["evals_ch"], "mu": s["evals_mu"]}}))


if __name__ == "__main__":
    main()
