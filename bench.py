#!/usr/bin/env python
"""Benchmark: TPSC solves/s on one B200 (or N independent replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one full TPSC solve of the 256x256 lattice with 2048 positive
fermionic Matsubara frequencies (Nw0 = 4096; t' = -0.15, U = 4, n = 0.875,
T = 0.05): chi0 -> Usp, Uch (sum-rule roots) -> V(r, tau) -> Sigma(k, i w_n)
-> Tr Sigma G -> mu (root of Tr(G - G0)) -> Tr Sigma G at mu.  The inputs are
model parameters (synthetic; no dataset exists for this path).

* value: device-resident solves/s of the mixed-precision + Newton form
  (FP32 G, chi0 and V slice transforms; FP64 for the rest), Sigma compared
  with the FP64 forms' (reported), each step timed with CUDA events on the
  library's own stream, L2 flushed (512 MB write) before every step; with
  N > 1 every rank solves its own replica (weak scaling, no collective on the
  data path) and the time is the max over ranks.
* e2e: the same solve through the public API with the model's lattice tables
  copied host->device and the self-energy Sigma(k, i w_n) (S, C2, C3, C4) and
  scalars copied device->pinned host inside the timed region; each step's
  copy overlaps the next step's compute.  Sigma comes back in the mixed
  form's own precision, formed in FP64 and rounded to FP32
  (tpsc_get_sigma32_async, 137 MB); the FP64 copy of S and its tails
  (tpsc_get_self_async, 275 MB) is timed and reported beside it.
* roofline: every stage kernel re-launched alone and timed with CUDA events;
  the dominant one (largest share of a solve) against the measured HBM copy
  bandwidth.
* cpu_baseline / --impl reference: the reference's own code (oracle/_ref,
  compiled from the unmodified sources) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(nk0=256, Nw0=4096, U=4.0, tp=-0.15, tpp=0.0, t3=0.0, n=0.875, T=0.05)
WORKLOAD_NAME = ("TPSC solve, 256x256 lattice, 2048 positive fermionic iwn (Nw0=4096), "
                 "t'=-0.15, U=4, n=0.875, T=0.05")
METRIC = "TPSC solves/s at 256²×2048 iωn: mixed+Newton vs FP64 GPU at ≤1e-6 ΔΣ; HBM GB/s"
PROBE = os.path.join(ROOT, "oracle", "_ref", "tpsc_ref_probe")
FALLBACK_HBM = 6650.0


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "samples": len(rows), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# reference CPU code
# ---------------------------------------------------------------------------
def run_reference_once(threads: int):
    """One solve by the reference binary; returns (seconds per solve without the
    half-grid pre-pass, raw seconds with it)."""
    if not os.path.exists(PROBE):
        raise RuntimeError("oracle/_ref/tpsc_ref_probe is missing (make -C oracle/ref)")
    w = WORKLOAD
    with tempfile.TemporaryDirectory() as d:
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        args = [PROBE, d, "bench"] + [repr(w[k]) for k in ("U", "tp", "tpp", "t3", "n", "T")] + [
            str(w["nk0"]), str(w["Nw0"])]
        subprocess.run(args, check=True, env=env, stdout=subprocess.DEVNULL)
        meta = {}
        for line in open(os.path.join(d, "meta.txt")):
            p = line.split()
            if len(p) >= 2:
                meta[p[0]] = p[1]
    raw = float(meta["t_self"]) + float(meta["t_traceSelfG"]) + float(meta["t_find_mu"])
    return raw - float(meta["t_half"]), raw


def reference_arm(a, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    budget = 200.0
    times, raws = [], []
    t_start = time.time()
    # warm-up: at most one (the reference has no caches to warm)
    if a.warmup > 0:
        run_reference_once(threads)
    for _ in range(a.steps):
        t, r = run_reference_once(threads)
        times.append(t)
        raws.append(r)
        if time.time() - t_start > budget:
            break
    sec = sum(times) / len(times)
    value = 1.0 / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": len(times), "warmup": min(a.warmup, 1), "ms_per_step": 1e3 * sec, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "form": "reference C++ (OpenMP), unmodified sources",
                   "parallelism": "replicas"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(times)} full solves of the workload (steps capped by a "
                                   f"{budget:.0f}s budget); half-grid Usp/Uch pre-pass timed alone and "
                                   "subtracted; the reference's own file writes included; FFTW replaced "
                                   "by this repo's FFTW-API shim"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "raw_seconds_with_prepass": sum(raws) / len(raws),
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def our_arm(a, world, rank, local_rank):
    import ctypes as C

    import numpy as np
    import torch

    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Context, Green

    dev = local_rank
    torch.cuda.set_device(dev)
    ctx = Context(dev)
    w = WORKLOAD
    g = Green(w["nk0"], w["Nw0"], w["n"], w["T"], 0.1, (w["tp"], w["tpp"], w["t3"], w["U"]), ctx=ctx)
    sp = C.c_void_p()
    ctx.call("tpsc_get_stream", C.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value, device=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def launches():
        c = C.c_longlong()
        ctx.call("tpsc_launch_count", C.byref(c))
        return c.value

    def timed_solves(form):
        """K solves of one root-search form, each bracketed by CUDA events on
        the library stream after an L2 flush; returns total ms (max over
        ranks), kernels launched, the clock record, scalars and stage times."""
        g.set_form(form)
        # the clock sampler starts before the warm-up so that it is running
        # (nvidia-smi takes a moment to start) when the timed steps begin
        with ClockSampler(dev) as clk:
            for _ in range(a.warmup):
                g.solve()
            torch.cuda.synchronize()
            barrier(world)
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(a.steps)]
            l0 = launches()
            torch.cuda.synchronize()
            for i in range(a.steps):
                flush.zero_()
                torch.cuda.synchronize()
                ev[i][0].record(stream)
                g.solve()
                ev[i][1].record(stream)
            torch.cuda.synchronize()
        n = launches() - l0
        t = allreduce_max(sum(s.elapsed_time(e) for s, e in ev), world, dev)
        return t, n, clk.summary(), g.scalars(), g.stage_times()

    # ---- the tau transforms' tiling for this shape, picked by timing both
    # (tpsc_tune_tau_tiles: one column pair or four columns per CTA) ----------
    g.set_form(_lib.FORM_NEWTON | _lib.FORM_MIXED)
    g.solve()
    tile_ms = np.zeros(6)
    ctx.call("tpsc_tune_tau_tiles", 5, tile_ms.ctypes.data_as(C.POINTER(C.c_double)))
    tau_tiles = {kind: {"pair_ms": float(tile_ms[2 * k]), "quad_ms": float(tile_ms[2 * k + 1]),
                        "picked": "pair" if tile_ms[2 * k] <= tile_ms[2 * k + 1] else "quad"}
                 for k, kind in enumerate(("chi0_tau", "vertex_tau", "sigma_tau"))}
    # ---- the FP32 slice transforms' plan for this lattice, picked by timing
    # every plan each kind supports (tpsc_tune_slice_plans: packed FFTs, the
    # folded matrix DCT-I on the FP32 pipe, the same on the tensor cores) ------
    g.solve()
    plan_ms = np.zeros(12)
    plan_names = ("fft", "matrix_fp32", "matrix_tensor_3xtf32")
    slice_plans = {}
    try:
        ctx.call("tpsc_tune_slice_plans", 5, plan_ms.ctypes.data_as(C.POINTER(C.c_double)))
    except Exception as ex:  # keep the library's default plans and say why
        for k in range(4):
            _lib.load().tpsc_set_slice_plan(k, w["nk0"], 0)
        slice_plans["tuner_error"] = str(ex)
    for k, kind in enumerate(("gslice", "chi0_slice", "vertex_q", "sigma_slice")):
        slice_plans[kind] = {plan_names[pl] + "_ms": float(plan_ms[3 * k + pl])
                             for pl in range(3) if plan_ms[3 * k + pl] > 0}
        slice_plans[kind]["picked"] = plan_names[_lib.load().tpsc_get_slice_plan(k, w["nk0"])]

    # ---- device-resident solves: the FP64 drop-in with the reference's root
    # searches, the FP64 Newton form, then mixed precision + Newton (the
    # headline); Sigma of the two Newton forms compared ------------------------
    ms_ref, _, _, sc_ref, stages_ref = timed_solves(_lib.FORM_REFERENCE)
    ms_n64, _, _, sc_n64, stages_n64 = timed_solves(_lib.FORM_NEWTON)
    sigma64 = g.sigma()
    MIXED = _lib.FORM_NEWTON | _lib.FORM_MIXED
    ms, n_launch, clocks, sc, stages = timed_solves(MIXED)
    graph_stats = g.graph_stats()
    dsigma = float(np.max(np.abs(g.sigma() - sigma64)) / np.max(np.abs(sigma64)))
    del sigma64
    value = world * a.steps / (ms / 1e3)
    value_ref = world * a.steps / (ms_ref / 1e3)
    value_n64 = world * a.steps / (ms_n64 / 1e3)

    # ---- end to end through the public API: every step sets the model (its
    # lattice tables go host -> device), solves and copies Sigma (S, C2, C3,
    # C4: 275 MB) and the scalars back to pinned host memory.  The copy of
    # step i runs on the library's copy stream while step i + 1 computes
    # (tpsc_get_self_async, two alternating pinned buffers); the timed region
    # ends after the last copy.  The working set (~2.4 GB) exceeds L2, so no
    # flush is needed between steps. ---------------------------------------------
    nk0, nw0, nbk, n8 = g.dims()
    # Sigma(k, i w_n) copied out in FP32 (the mixed form's own precision,
    # 137 MB; tpsc_get_sigma32_async) and, for comparison, S in FP64 (275 MB)
    bufs = {}
    for f32 in (True, False):
        bufs[f32] = []
        for _ in range(2):
            S_host = torch.empty((nw0 // 2, n8, 2), dtype=torch.float32 if f32 else torch.float64).pin_memory()
            S_host = S_host.numpy().view(np.complex64 if f32 else np.complex128)[..., 0]
            v = [torch.empty(n8, dtype=torch.float64).pin_memory().numpy() for _ in range(3)]
            bufs[f32].append((S_host, v))
    h2d = 2 * n8 * 8

    def d2h_bytes(f32):
        return bufs[f32][0][0].nbytes + (0 if f32 else 3 * n8 * 8) + len(_lib.SCALARS) * 8

    def e2e_steps(k, f32):
        for i in range(k):
            g2 = Green(w["nk0"], w["Nw0"], w["n"], w["T"], 0.1, (w["tp"], w["tpp"], w["t3"], w["U"]), ctx=ctx)
            g2.set_form(MIXED)
            g2.solve()
            S_c, v = bufs[f32][i % 2]
            if f32:
                g2.sigma_async32(S_c)
            else:
                g2.self_energy_async(S_c, *v)
            g2.scalars()
        g2.wait_copies(join_stream=True)

    def e2e_run(f32):
        # timed with direct launches (graph mode 1: every step is a new model)
        # and with every solve captured and its graph updated in place (mode
        # 2); the faster counts, both are reported
        modes = {}
        for mode in (1, 2):
            g.set_graph_mode(mode)
            e2e_steps(2, f32)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            e2e_steps(a.steps, f32)
            e1.record(stream)
            torch.cuda.synchronize()
            g.wait_copies()
            modes[mode] = world * a.steps / (allreduce_max(e0.elapsed_time(e1), world, dev) / 1e3)
        g.set_graph_mode(1)
        return modes

    e2e_modes = e2e_run(True)
    e2e_modes64 = e2e_run(False)
    e2e_mode = max(e2e_modes, key=e2e_modes.get)
    e2e = e2e_modes[e2e_mode]
    d2h = d2h_bytes(True)

    # ---- per-kernel timing (stages re-launched alone, in order, as the
    # mixed + Newton solve runs them) -------------------------------------------
    g.set_form(MIXED)
    g.solve()
    torch.cuda.synchronize()
    reps = 3
    per = {}
    for rep in range(reps):
        for k, name in enumerate(_lib.KERNELS):
            if name == "chi0_slice+tau":
                continue
            flush.zero_()
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            ctx.call("tpsc_run_kernel", k)
            e.record(stream)
            torch.cuda.synchronize()
            per.setdefault(name, []).append(s.elapsed_time(e))
    per_ms = {k: min(v) for k, v in per.items()}
    per_ms["mu_roots"] = per_ms.pop("sigma_moments+mu_roots") - per_ms["sigma_moments"]
    # launches per mixed + Newton solve: the root searches run inside the two
    # cooperative root kernels; the single full and Newton-form evaluations
    # (sumrule, trace_diff_G and their _newton forms) are timed for reference
    # but not launched by a solve
    counts = {k: 1 for k in per_ms}
    for k in ("sumrule", "trace_diff_G", "sumrule_newton", "trace_diff_G_newton"):
        counts[k] = 0
    share = {k: per_ms[k] * counts[k] for k in per_ms}
    dom = max(share, key=share.get)

    def kernel_bytes(name):
        kb = C.c_double()
        if name == "mu_roots":
            ctx.call("tpsc_kernel_bytes", _lib.KERNELS.index("sigma_moments+mu_roots"), C.byref(kb))
            b = kb.value
            ctx.call("tpsc_kernel_bytes", _lib.KERNELS.index("sigma_moments"), C.byref(kb))
            return b - kb.value
        ctx.call("tpsc_kernel_bytes", _lib.KERNELS.index(name), C.byref(kb))
        return kb.value

    kb = C.c_double(kernel_bytes(dom))
    achieved = kb.value / (per_ms[dom] / 1e3) / 1e9
    peak, peak_kind = measured_hbm()
    slice_kind = {"gslice": 0, "chi0_slice": 1, "vertex_q": 2, "sigma_slice": 3}
    dom_plan = _lib.load().tpsc_get_slice_plan(slice_kind[dom], w["nk0"]) if dom in slice_kind else 0
    traffic = profiled_traffic(dom, dom_plan)

    # ---- the batched parameter sweep (512 seeded points, uneven lattices and
    # cutoffs), mixed + Newton, on the tuned number of solver streams --------
    batch = None
    if world == 1 and not a.no_batch:
        batch = batch_sweep(a.steps)
    extra = None
    if world == 1 and not a.no_extra:
        extra = extra_configs()

    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (model parameters; no dataset)",
        "config": {"workload": WORKLOAD_NAME,
                   "form": "mixed precision (FP32 slice transforms of G, chi0, V and Sigma on the autotuned "
                           "slice plan, Sigma's near field |r| <= 4 in FP64; FP64 tau transforms, sums, roots) "
                           "+ Newton root searches with moment series",
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "512 MB flush before every step; working set ~2.4 GB per solve",
                   "sumrule_evals": int(sc["evals_sp"] + sc["evals_ch"]), "mu_evals": int(sc["evals_mu"]),
                   "launch": "Newton-form solves replay one captured CUDA graph (tpsc_set_graph_mode 1: "
                             "same kernels and arguments as direct launches); the FP64 drop-in with the "
                             "reference's root searches runs direct launches with its host round trips"},
        "solve_graph": graph_stats,
        "tau_tiles": tau_tiles,
        "slice_plans": slice_plans,
        "forms": {"mixed_newton": {"solves_per_s": value, "ms_per_step": ms / a.steps, "stage_ms": stages,
                                   "max_rel_dSigma_vs_fp64": dsigma},
                  "fp64_newton": {"solves_per_s": value_n64, "ms_per_step": ms_n64 / a.steps,
                                  "stage_ms": stages_n64},
                  "fp64_reference_roots": {"solves_per_s": value_ref, "ms_per_step": ms_ref / a.steps,
                                           "stage_ms": stages_ref,
                                           "sumrule_evals": int(sc_ref["evals_sp"] + sc_ref["evals_ch"]),
                                           "mu_evals": int(sc_ref["evals_mu"])},
                  "mixed_newton_over_fp64_reference_roots": value / value_ref,
                  "max_rel_diff_roots_fp64_newton": max(abs(sc_n64[k] - sc_ref[k]) / abs(sc_ref[k])
                                                        for k in ("Usp", "Uch", "mu")),
                  "max_rel_diff_roots_mixed": max(abs(sc[k] - sc_ref[k]) / abs(sc_ref[k])
                                                  for k in ("Usp", "Uch", "mu"))},
        "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "graph_mode": e2e_mode, "solves_per_s_by_graph_mode": {str(k): v for k, v in e2e_modes.items()},
                "copied": "Sigma(k, i w_n) formed in FP64 on the device, rounded to FP32 "
                          "(tpsc_get_sigma32_async; within the mixed form's 1e-6 bound, tests/test_gpu_async.py)",
                "fp64_S_copy": {"value": max(e2e_modes64.values()), "d2h_bytes_per_step": d2h_bytes(False),
                                "solves_per_s_by_graph_mode": {str(k): v for k, v in e2e_modes64.items()}}},
        "roofline": {"bound": "hbm", "kernel": dom, "slice_plan": dom_plan, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "algorithmic_bytes": kb.value, "launch_ms": per_ms[dom]},
        "kernels_ms": per_ms, "kernel_launches_per_solve": counts, "stage_ms": stages,
        "gpu_launches": n_launch,
        "clocks": clocks,
        "results": {k: sc[k] for k in ("Usp", "Uch", "dblOcc", "mu", "Sigma_inf")},
    }
    if batch is not None:
        line["batch"] = batch
    if extra is not None:
        line["configs"] = extra
    if world == 1 and not a.no_cpu_baseline:
        try:
            t, raw = run_reference_once(os.cpu_count() or 1)
            line["cpu_baseline"] = {
                "value": 1.0 / t, "unit": "solves/s", "cores": os.cpu_count() or 1, "kind": "reference",
                "sample": "one full solve of the same workload by the reference binary (half-grid pre-pass "
                          f"subtracted, {raw:.1f}s raw)"}
        except Exception as ex:  # the binary travels with the tree; report if it does not
            line["cpu_baseline"] = {"value": None, "unit": "solves/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {ex}"}
    print(json.dumps(line), flush=True)


def batch_sweep(steps):
    """The 512-point sweep through the batched sweep API: tuned stream count
    (1, 2, 4, 8, 16 contexts timed on the sweep), then the sweep timed on that
    count (best of a few calls).  Wall time from a device-idle start to a
    device-idle end, host work included."""
    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import Batch, sweep_points

    pts = sweep_points(512, seed=20261203)
    form = _lib.FORM_NEWTON | _lib.FORM_MIXED
    b = Batch(nstreams=1)
    tune = b.tune(pts, form, max_streams=16)
    # the sweep as direct launches (graph mode 0), as one graph launch per
    # point (mode 2: each grid's graph updated in place for the point) and by
    # shape groups (mode 3: one launch per stage over every point of a
    # (nk0, Nw0) group, one graph launch per group, tpsc_solve_points)
    per_mode = {}
    st = None
    for mode in (0, 2, 3):
        b.set_graph_mode(mode)
        b.solve(pts, form)  # mode 2: every grid captured once before timing
        times = []
        for _ in range(max(1, min(steps, 5))):
            _, st, ms = b.solve(pts, form)
            times.append(ms)
        per_mode[mode] = times
    nfail = int((st != 0).sum())
    mode = min(per_mode, key=lambda m: min(per_mode[m]))
    best = min(per_mode[mode])
    shapes = sorted({(int(p[0]), int(p[1])) for p in pts})
    out = {"workload": "512 solves from tpsc_sweep_points(seed 20261203): nk0 in {32,64,128,256}, U~U[1,6], "
                       "n~U[0.7,1], log T~U[ln .03, ln .5], t'~U[-.3,0], Nw0 = 2 nextpow2(ceil(40/(pi T)))",
           "form": "mixed + Newton", "shapes": len(shapes), "streams": b.nstreams,
           "solves_per_s": 512 / (best / 1e3), "ms_per_sweep": best, "graph_mode": mode,
           "ms_per_sweep_direct": per_mode[0], "ms_per_sweep_graphs": per_mode[2],
           "ms_per_sweep_shape_groups": per_mode[3],
           "launches": {"0": "every kernel of every point", "2": "one graph per point",
                        "3": "one graph per (nk0, Nw0) group, each kernel over all its points"},
           "sequential_solves_per_s": 512 / (tune[1] / 1e3), "tune_ms": tune, "failed_points": nfail,
           "timing": "host wall clock around the whole call, device idle at both ends"}
    b.close()
    return out


def extra_configs():
    """The other workloads of the measurement plan, each timed once after a
    warm-up run (host wall clock, device idle at both ends, ms):
    config 1, plain FP64 TPSC at 32^2 x 256 positive iwn with chi_jj for 16
    bosonic frequencies and the Pade spectral weight of every k on 1000 real
    frequencies; config 3, the optical conductivity at 128^2 x 1024 positive
    iwn, mixed + Newton, sigma(iq_n) n = 1..256 against the FP64 form, Pade of
    sigma on 2000 frequencies; config 4, the sum-rule sensitivities
    d(Usp, Uch, D)/d(U, mu, t') at 128^2 x 1024."""
    import numpy as np
    import torch

    from tpsc_conductivity_b200 import _lib
    from tpsc_conductivity_b200.api import CondOpt, Green

    def timed(f):
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = f()
        torch.cuda.synchronize()
        return r, 1e3 * (time.perf_counter() - t)

    out = {}
    # config 1
    c = CondOpt(32, 512, 0.875, 0.25, 0.05, (0.0, 0.0, 0.0, 2.0))
    c.set_form(_lib.FORM_REFERENCE)
    w1 = np.linspace(-8.0, 8.0, 1000) + 0.05j

    def c1():
        ms = {}
        _, ms["solve"] = timed(c.solve)
        _, ms["chijj"] = timed(lambda: c.calc_chijj_vertex_corr_all_optim(False, 3, 1))
        s16, ms["sigma_iqn"] = timed(lambda: c.sigma_qn(16))
        sa, ms["pade"] = timed(lambda: c.pade_sigma(w1, Nn=32))
        return s16, sa, ms

    c1()
    (s16, _), (_, A), ms1 = c1()
    sc = c.scalars()
    out["c1_l32_w512_plain_fp64"] = {
        "ms": ms1, "Usp": sc["Usp"], "Uch": sc["Uch"], "dblOcc": sc["dblOcc"],
        "sigma_iq1": float(s16[0]), "pade": "Sigma(k, w + 0.05i) and A(k, w) for all 153 octant k, 1000 w in "
                                              "[-8, 8], 32 Matsubara nodes",
        "A_finite": bool(np.all(np.isfinite(A)))}
    # config 3
    w3 = np.linspace(0.0, 10.0, 2000)

    def c3(g):
        ms = {}
        _, ms["solve"] = timed(g.solve)
        _, ms["chijj"] = timed(lambda: g.calc_chijj_vertex_corr_all_optim(False, 3, 1))
        sig, ms["sigma_iqn"] = timed(lambda: g.sigma_qn(256)[0])
        pade, ms["pade"] = timed(lambda: g.sigma_pade(w3, 64, 0.0)[0])
        return sig, pade, ms

    objs = {}
    for name, form in (("mixed_newton", _lib.FORM_NEWTON | _lib.FORM_MIXED), ("fp64_newton", _lib.FORM_NEWTON)):
        objs[name] = CondOpt(128, 2048, 0.9, 0.1, 0.1, (0.0, 0.0, 0.0, 3.0))
        objs[name].set_form(form)
        # two warm-up runs: the second solve of a model is captured as a
        # CUDA graph, the timed one replays it
        c3(objs[name])
        c3(objs[name])
    sig_m, pade_m, ms3 = c3(objs["mixed_newton"])
    st3 = objs["mixed_newton"].stage_times()
    sig_d, _, ms3d = c3(objs["fp64_newton"])
    # the chi_jj stage against the HBM roofline: device time of its kernels
    # (CUDA events around the slices, the tau kernel and the finish) and the
    # minimal-traffic model 8 K4 (Nw0+1) s + N8 Nb s + N8 (Nw0/2) 2s, s = 8 B
    nbk3, nw3 = 128 // 2 + 1, 2048
    K4, N8, Nb = (nbk3 - 2) * nbk3, nbk3 * (nbk3 + 1) // 2, nw3 // 2 + 1
    alg3 = 8.0 * (8 * K4 * (nw3 + 1) + N8 * Nb + N8 * (nw3 // 2) * 2)
    dev3 = st3["cond_slices"] + st3["cond_tau"] + st3["cond_finish"]
    peak3, _ = measured_hbm()
    # the Aslamazov-Larkin correction on the non-uniform grid of mmin = 3
    g3 = objs["fp64_newton"]
    g3.calc_chijj_vertex_corr_all_optim(True, 3, 1)
    al3, t_al = timed(lambda: g3.calc_chijj_vertex_corr_all_optim(True, 3, 1))
    out["c3_l128_w2048_conductivity"] = {
        "ms_mixed_newton": ms3, "ms_fp64_newton": ms3d,
        "max_rel_err_sigma_iqn_mixed_vs_fp64": float(np.max(np.abs(sig_m - sig_d)) / np.max(np.abs(sig_d))),
        "pade": "sigma(w) on 2000 w in [0, 10] from 64 bosonic nodes", "pade_finite": bool(np.all(np.isfinite(pade_m))),
        "chijj_roofline": {"bound": "hbm", "device_ms": dev3, "stage_ms": {k: st3[k] for k in
                                                                        ("cond_slices", "cond_tau", "cond_finish")},
                           "algorithmic_bytes": alg3, "achieved": alg3 / (dev3 * 1e-3) / 1e9, "peak": peak3,
                           "unit": "GB/s", "frac": alg3 / (dev3 * 1e-3) / 1e9 / peak3},
        "aslamazov_larkin": {"ms": t_al, "mmin": 3, "grid_frequencies": int(len(al3["ind_freq"])),
                             "ms_per_frequency": t_al / max(1, len(al3["ind_freq"]) - 1),
                             "note": "includes the bubble + Maki-Thompson call before it (FP64)"}}
    # config 4
    g4 = CondOpt(128, 2048, 0.85, 0.1, 0.1, (-0.2, 0.0, 0.0, 4.0))
    g4.set_form(_lib.FORM_NEWTON)
    g4.find_Usp_Uch_grid(128, 2048)
    g4.sumrule_tangents()
    J, t4 = timed(g4.sumrule_tangents)
    # sigma(iq1): the reverse pass (tpsc_sigma_iqn_bwd) after one solve +
    # chi_jj, and the central differences of full FP64 solves beside it
    g4.solve()
    g4.ctx.call("tpsc_chijj", 1)
    _, t4f = timed(lambda: (g4.solve(), g4.ctx.call("tpsc_chijj", 1)))
    g4.sigma_qn_vjp([1.0])
    (gr4, _), t4b = timed(lambda: g4.sigma_qn_vjp([1.0]))
    g4.sigma_qn_sensitivities(1)
    (ds4, dD4), t4s = timed(lambda: g4.sigma_qn_sensitivities(1))
    out["c4_l128_w2048_sensitivities"] = {
        "ms": t4, "d_dU": J["U"], "d_dmu": J["mu"], "d_dtp": J["tp"],
        "checked": "central differences, tests/test_gpu_tangent.py",
        "sigma_iq1": {"reverse_pass": {"ms": t4b, "d_dU": float(gr4[0]), "d_dmu": float(gr4[1]),
                                       "d_dtp": float(gr4[2]),
                                       "method": "tpsc_sigma_iqn_bwd: chi_jj, mu, Sigma, V backward (FP64) chained "
                                                 "with the chi0 and sum-rule forward tangents; "
                                                 "tests/test_gpu_adjoint.py"},
                      "forward_ms": t4f, "reverse_over_forward": t4b / t4f,
                      "central_differences": {"ms": t4s, "d_dU": float(ds4[0, 0]), "d_dmu": float(ds4[1, 0]),
                                              "d_dtp": float(ds4[2, 0]),
                                              "method": "six FP64 Newton solves + chi_jj, h = 1e-5, base point "
                                                        "solved again; tests/test_gpu_sigma_fd.py"},
                      "max_rel_diff": float(np.max(np.abs(gr4 - ds4[:, 0])) / np.max(np.abs(ds4[:, 0])))}}
    out["timing"] = "host wall clock around each call after a warm-up run, device idle at both ends"
    return out


def profiled_traffic(kernel, plan=0):
    """DRAM bytes per launch of `kernel` (slice kernels: under slice plan
    `plan`, listed as name@plan unless it is the FFT plan) from the committed
    ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    key = kernel if not plan else f"{kernel}@{plan}"
    try:
        for line in open(p):
            f = line.split()
            if len(f) >= 2 and f[0] == key:
                return float(f[1])
    except Exception:
        pass
    return None


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def allreduce_max(x, world, dev):
    """The max of x over the ranks (the replicas' slowest time).  dev: the
    rank's CUDA device (NCCL), or None for a host tensor (gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cpu" if dev is None else f"cuda:{dev}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-point batched sweep")
    ap.add_argument("--no-extra", action="store_true", help="skip the measurements of the other workloads")
    ap.add_argument("--nk0", type=int, default=None, help="lattice side override (profiling only)")
    ap.add_argument("--nw0", type=int, default=None, help="Nw0 override (profiling only)")
    a = ap.parse_args()
    if a.nk0 or a.nw0:
        global WORKLOAD_NAME
        WORKLOAD["nk0"] = a.nk0 or WORKLOAD["nk0"]
        WORKLOAD["Nw0"] = a.nw0 or WORKLOAD["Nw0"]
        WORKLOAD_NAME = f"PROFILING OVERRIDE nk0={WORKLOAD['nk0']} Nw0={WORKLOAD['Nw0']} (not the headline)"
        a.no_cpu_baseline = True
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and a.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if a.impl == "reference":
            reference_arm(a, world, rank)
        else:
            our_arm(a, world, rank, local_rank)
    finally:
        if world > 1 and a.impl == "ours":
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
