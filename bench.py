#!/usr/bin/env python
"""Benchmark of the B200 LEQ_BICGS path (MFIX SOLVE_LIN_EQ -> LEQ_BICGS).

Workload (default): one 256x256x256 7-point upwind convection-diffusion system
(258^3 = 17,173,512 cells with the wall layer), LINE preconditioner, RSRS sweeps,
TOL 1e-8, ITMAX 500, seeded synthetic data in the MFIX A_M/B_M layout.  A step is
one complete solve.  Reported:

* value      solves/s of the FP32-inner / FP64-refinement form, inputs resident in
             HBM (A_M is 0.96 GB, larger than L2, so nothing is cached between steps);
* fp64       the plain FP64 drop-in on the same system, for the mixed-vs-FP64 ratio;
* e2e        the same metric through the Fortran-convention entry point
             mfixgpu_solve_lin_eq_ with pinned host arrays, copies inside the timing;
* roofline   the J-line sweep kernel (the dominant kernel): algorithmic bytes per
             launch / average launch time from CUDA events over the timed steps;
* accuracy   each form's error against an FP64 solution refined to a true residual of
             1e-14 (long-double residuals), and its difference from the oracle's solution;
* cpu_baseline  one complete solve of the same system by the oracle (a C restatement of the
             reference's FP64 LEQ_BICGS with the reference's OpenMP loops), timed.

``--impl reference`` times that CPU implementation alone (rank 0), with all host cores:
each step is one complete solve.
Multi-GPU: every rank solves its own replica (the path shards by independent
systems; a single system fits one GPU), value = systems solved by all ranks / max
over ranks of the device time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOADS = {
    "conv_diff_256": dict(kind="conv_diff", dims=(256, 256, 256), seed=0, itmax=500, tol=1e-8),
    "conv_diff_64": dict(kind="conv_diff", dims=(64, 64, 64), seed=0, itmax=500, tol=1e-8),
    "conv_diff_192": dict(kind="conv_diff", dims=(192, 192, 192), seed=0, itmax=500, tol=1e-8),
    "pressure_192x384x192": dict(kind="pressure_like", dims=(192, 384, 192), seed=0, itmax=5000, tol=1e-8),
    # METHOD 5 (LEQ_CG, FP64): symmetric diffusion whose diagonal-scaled operator stays symmetric
    "cg_diffusion_256": dict(kind="cg", dims=(256, 256, 256), seed=0, itmax=500, tol=1e-8),
    # 512 independent convection-diffusion systems, per-axis sizes U{16..96}, seeds 0..511
    "batch_512": dict(kind="batch", count=512, seed=0, itmax=500, tol=1e-8),
    # its first 64 systems (1.25e7 cells): the profiling case of the batched kernels
    "batch_64": dict(kind="batch", count=64, seed=0, itmax=500, tol=1e-8),
    # Poisson request stream: sizes log-uniform per axis on [24, 160], 20% pressure-like,
    # TOL from {1e-6, 1e-8}, 150 GB HBM admission budget
    "serve_poisson": dict(kind="serve", rate=2000.0, seconds=60.0, pool=1024, seed=0, budget=150e9),
}
DEFAULT_WORKLOAD = "conv_diff_256"

BYTES_FP64_ITER = 576  # algorithmic bytes per cell per BiCGSTAB iteration, FP64 (72 words)
BYTES_FP32_ITER = 288  # the same in the FP32 inner solve
BYTES_OUTER = 104      # FP64 refinement step: r = b - A x (80) + x update (24)
# a deflated FP32 iteration (near-singular systems) also reads z in the P, S and X
# updates (1 B each) and A z in both matvecs (4 B each)
BYTES_DEFL_ITER = 11
BYTES_DEFL_SETUP = 61  # z (1) written; A z from the FP64 diagonals (56) and z, written (4)
BYTES_SETUP = 128      # unit scaling (16 w) of FP64 A and B
# Algorithmic bytes per cell of one launch of each kernel class (FP32 inner form,
# FP64 drop-in): operands read + results written, reductions fused.
CLASS_BYTES = {
    "jline": (20, 40),          # half the cells: 3 factors + 4 off-line diagonals + rhs + old + new
    "p_update": (16, 32),       # R, P, V in, P out
    "matvec_alpha": (40, 80),   # 7 diagonals, x, Rtilde in, V out
    "s_update": (12, 24),       # R, V in, S out
    "matvec_omega": (40, 80),   # 7 diagonals, x, S in, T out
    "xr_update": (40, 64),      # FP32: x64 in/out (16), Phat, Shat, S, T, Rtilde in, R out
    "outer_step": (80, 80),     # FP64 A (56), x64, B in; FP32 R, Rtilde out
}


def true_rel_resid(s, x, rows: str = "max") -> float:
    """||B - A x|| / ||B|| of the row-scaled system, in numpy (x0 = 0, so ||B|| is the
    initial residual).  rows = "max": rows divided by max |A(ijk,:)| as BiCGSTAB
    scales them; "diag": divided by A(ijk,0) as CG does.  Host arrays as the caller
    passed them (unscaled)."""
    from mfix_b200 import systems as S

    m = np.abs(s.a).max(axis=0) if rows == "max" else s.a[3]
    a = s.a / m
    b = s.b / m
    r = b - S.matvec_np(s.imax2, s.jmax2, s.kmax2, s.do_k, a, x)
    return float(np.linalg.norm(r) / np.linalg.norm(b))


def work_launches(inner: int, outer: int, jline_per_iter: int = 8) -> dict:
    """Launches of each kernel class that did work in one solve.  The host polls
    convergence every few iterations, so some launches run after a system is
    done, and in the mixed form the inner-iteration kernels idle while an FP64
    update runs; those launches return at once and carry no algorithmic bytes."""
    w = {k: inner for k in CLASS_BYTES}
    w["jline"] = jline_per_iter * inner
    w["outer_step"] = outer
    return w


def class_table(kt: dict, cells: int, fp32: bool, peak: float, work: dict) -> dict:
    """Per kernel class: total ms over all launches, launches, launches that did
    work, mean us per working launch, achieved GB/s of algorithmic bytes over the
    total time, fraction of peak."""
    out = {}
    for name, (ms, n) in kt.items():
        if n == 0:
            continue
        nw = min(int(work.get(name, n)), int(n))
        row = {"ms": round(ms, 3), "launches": int(n), "work_launches": nw,
               "us_per_launch": round(1e3 * ms / max(nw, 1), 2)}
        if name in CLASS_BYTES:
            b = CLASS_BYTES[name][0 if fp32 else 1] * cells
            gbs = b * nw / (ms / 1e3) / 1e9 if ms > 0 else 0.0
            row.update({"gbs": round(gbs, 1), "frac": round(gbs / peak, 3)})
        out[name] = row
    return out


def _gen_system(spec):
    """One system of a batch or request pool (run in spawned worker processes)."""
    from mfix_b200 import systems as S

    kind, dims, tol, seed = spec
    return S.make_request_system(kind, dims, tol, seed)


def generate_systems(specs):
    """Seeded systems generated in parallel by spawned processes (before any GPU call)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    workers = max(1, min(32, (os.cpu_count() or 2) - 1))
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_gen_system, specs, chunksize=max(1, len(specs) // (4 * workers))))


def make_system(name: str):
    from mfix_b200 import systems as S

    w = WORKLOADS[name]
    i, j, k = w["dims"]
    if w["kind"] == "conv_diff":
        return S.conv_diff(i, j, k, seed=w["seed"], itmax=w["itmax"], tol=w["tol"])
    if w["kind"] == "cg":
        return S.diffusion_sym(i, j, k, seed=w["seed"], itmax=w["itmax"], tol=w["tol"])
    return S.pressure_like(i, j, k, seed=w["seed"], itmax=w["itmax"], tol=w["tol"])


def measured_peak_hbm() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel_file: str):
    """dram bytes per launch recorded from an ncu capture (profiles/), or None."""
    p = os.path.join(ROOT, "profiles", kernel_file)
    try:
        with open(p) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm.append(float(parts[1]))
                        smax = max(smax, float(parts[2]))
                    except ValueError:
                        continue
                    for nm, v in zip(names, parts[5:9]):
                        if v.lower().startswith("active"):
                            reasons.add(nm)
        except (OSError, TypeError):
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_solve(sys0) -> tuple:
    """One complete solve of the system by the oracle (the reference's FP64
    LEQ_BICGS restated in C, with the reference's OpenMP loops), timed; returns
    (seconds, the solved copy with its unit-scaled A/B, the oracle's stats)."""
    import oracle as O

    s = sys0.copy()
    t0 = time.perf_counter()
    st = O.leq_bicgs(s)
    return time.perf_counter() - t0, s, st


def accuracy(ref, st_ref, xs: dict) -> dict:
    """Errors of each solution in `xs` against the FP64 truth: the oracle's solution
    refined until ||b - A x|| <= 1e-14 ||b|| (x0 = 0, so ||b|| is the initial
    residual) with long-double residuals, on the unit-scaled system `ref`."""
    import oracle as O

    r0 = O.true_resid(ref, np.zeros(ref.n))
    t0 = time.perf_counter()
    x_truth, rel = O.truth_from(ref, ref.x, r0, rtol=1e-14)
    t_truth = time.perf_counter() - t0
    nt = float(np.linalg.norm(x_truth))
    no = float(np.linalg.norm(ref.x))
    out = {"truth_rel_resid": rel, "truth_s": t_truth,
           "oracle": {"iterations": st_ref["iterations"], "true_rel_resid": O.true_resid(ref, ref.x) / r0,
                      "err_vs_truth": float(np.linalg.norm(ref.x - x_truth)) / nt}}
    for name, x in xs.items():
        out[name] = {"err_vs_truth": float(np.linalg.norm(x - x_truth)) / nt,
                     "rel_diff_vs_oracle": float(np.linalg.norm(x - ref.x)) / no,
                     "true_rel_resid": O.true_resid(ref, x) / r0}
    return out


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_reference(args) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    w = args.workload
    if WORKLOADS[w]["kind"] in ("batch", "serve"):
        return run_reference_sample(args)
    if WORKLOADS[w]["kind"] == "cg":
        return run_reference_cg(args)
    import oracle as O

    sys0 = make_system(w)
    for _ in range(args.warmup):
        cpu_solve(sys0)
    times, its = [], 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        dt, _, st = cpu_solve(sys0)
        times.append(dt)
        its = st["iterations"]
    wall = time.perf_counter() - t0
    v = args.steps / sum(times)
    sample = (f"{args.steps} complete oracle solves of the {sys0.imax2}x{sys0.jmax2}x{sys0.kmax2}-cell system "
              f"({its} iterations each), one per step")
    line = {"impl": "reference", "metric": "solves/s", "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(w, sys0),
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall, "iterations": its,
            "cpu_gbs": BYTES_FP64_ITER * its * sys0.n / (sum(times) / args.steps) / 1e9}
    print(json.dumps(line), flush=True)


def run_reference_cg(args) -> None:
    """CPU arm of the CG workload: complete oracle LEQ_CG solves, one per step."""
    import oracle as O

    w = args.workload
    sys0 = make_system(w)
    vals, its = [], 0
    for step in range(args.warmup + args.steps):
        s = sys0.copy()
        t0 = time.perf_counter()
        st = O.leq_cg(s)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            vals.append(1.0 / dt)
            its = st["iterations"]
    v = float(np.mean(vals))
    sample = f"{args.steps} complete oracle CG solves of the {w} system ({its} iterations each)"
    line = {"impl": "reference", "metric": "solves/s", "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w, "grid": list(WORKLOADS[w]["dims"]), "cells": sys0.n, "method": 5},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference_sample(args) -> None:
    """CPU arm of the batched and serving workloads: the oracle solves whole
    systems of the batch (or of the serving pool, at the pool's TOL) for a
    bounded time per step."""
    import oracle as O
    from mfix_b200 import systems as S

    w = WORKLOADS[args.workload]
    if w["kind"] == "batch":
        specs = [("conv_diff", d, w["tol"], q) for q, d in enumerate(S.batch_sizes(w["count"], w["seed"]))]
    else:
        specs = S.serve_mix(w["pool"], w["seed"])
    vals, k_tot = [], 0
    for step in range(args.warmup + args.steps):
        dt, k = 0.0, 0
        while k < len(specs) and (k < 2 or dt < 10.0):
            c = _gen_system(specs[(step * 7 + k) % len(specs)])  # generation is outside the timing
            t1 = time.perf_counter()
            O.leq_bicgs(c)
            dt += time.perf_counter() - t1
            k += 1
        if step >= args.warmup:
            vals.append(k / dt)
            k_tot += k
    v = float(np.mean(vals))
    sample = f"{k_tot} whole systems of the {args.workload} workload solved by the oracle over {args.steps} steps"
    line = {"impl": "reference", "metric": "solves/s", "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(w: str, s) -> dict:
    return {"workload": w, "grid": list(WORKLOADS[w]["dims"]), "cells": s.n, "pc": "LINE", "sweep": "RSRS",
            "tol": WORKLOADS[w]["tol"], "itmax": WORKLOADS[w]["itmax"], "batch": 1,
            "l2_policy": "inputs larger than L2 (A_M 7*8*cells bytes), no flush needed"}


def pressure_measure(dev, steps: int, warmup: int) -> dict:
    """The pressure-correction-like system (192x384x192 interior cells, symmetric
    diffusion with void-fraction-weighted faces, diagonal excess 1e-6): the FP64
    drop-in and the mixed form (deflated) on the device-resident arrays; solves/s,
    iterations, FP64 true residual of the scaled system, and the measured
    coefficient contrast."""
    import torch

    from mfix_b200 import leq
    from mfix_b200 import systems as S

    name = "pressure_192x384x192"
    t0 = time.perf_counter()
    s = make_system(name)
    t_gen = time.perf_counter() - t0
    n = s.n
    A0 = torch.from_numpy(s.a).to(dev)
    B0 = torch.from_numpy(s.b).to(dev)
    A, B = torch.empty_like(A0), torch.empty_like(B0)
    X = torch.zeros(n, dtype=torch.float64, device=dev)
    geom = leq.geom(s.imax2, s.jmax2, s.kmax2, s.do_k)

    def solve(precision):
        A.copy_(A0)
        B.copy_(B0)
        X.zero_()
        torch.cuda.synchronize()
        rc, res = leq.batch_solve([s], precision=precision, on_device=True,
                                  pointers=[(A.data_ptr(), B.data_ptr(), X.data_ptr())])
        if rc != 0 or res[0].ier != 0:
            raise RuntimeError(f"pressure solve rc={rc} ier={res[0].ier if res else None}: {leq.last_error()}")
        return res[0], leq.last_stats()

    def true_rel():
        y = torch.empty_like(X)
        leq.leq_matvec(geom, A.data_ptr(), X.data_ptr(), y.data_ptr())
        return float(torch.linalg.vector_norm(B - y) / torch.linalg.vector_norm(B))

    peak, peak_kind = measured_peak_hbm()
    out = {"workload": name, "grid": list(WORKLOADS[name]["dims"]), "cells": n, "tol": s.tol,
           "coefficient_contrast": S.coefficient_contrast(s), "generation_s": t_gen, "steps": steps}
    xs = {}
    for form, prec in (("fp64", 0), ("mixed", 1)):
        for _ in range(warmup):
            solve(prec)
        ms = []
        for _ in range(steps):
            r, st = solve(prec)
            ms.append(st["device_ms"])
        t = float(np.mean(ms))
        if prec == 0:
            alg = n * (r.iterations * BYTES_FP64_ITER + BYTES_SETUP + 80)
        else:
            per = BYTES_FP32_ITER + (BYTES_DEFL_ITER if st["deflated"] else 0)
            alg = n * (r.iterations * per + r.outer_steps * BYTES_OUTER + BYTES_SETUP + 7 * 12 +
                       (BYTES_DEFL_SETUP if st["deflated"] else 0))
        out[form] = {"solves_per_s": 1e3 / t, "ms_per_solve": t, "iterations": r.iterations,
                     "outer_steps": r.outer_steps, "fp64_fallback": r.fp64_fallback, "deflated": st["deflated"],
                     "true_rel_resid": true_rel(), "alg_gbs": alg / (t / 1e3) / 1e9,
                     "frac_of_peak": alg / (t / 1e3) / 1e9 / peak, "gpu_launches": st["kernel_launches"]}
        xs[form] = X.clone()
    out["mixed_vs_fp64"] = out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"]
    out["mixed"]["rel_diff_vs_fp64"] = float(torch.linalg.vector_norm(xs["mixed"] - xs["fp64"]) /
                                             torch.linalg.vector_norm(xs["fp64"]))
    out["peak_gbs"], out["peak_kind"] = peak, peak_kind
    return out


def run_legs(args, dev) -> dict:
    """The other benchmark configurations, measured in the default run: the
    pressure-like system, the 512-system batch and a serving run; each with the
    clocks seen during it, or the error that stopped it."""
    import torch

    legs = {}
    want = [x for x in args.legs.split(",") if x]

    def leg(name, fn):
        sampler = ClockSampler(dev.index or 0)
        t0 = time.perf_counter()
        try:
            with sampler:
                r = fn()
            r["clocks"] = sampler.summary()
        except Exception as e:  # a failed leg is reported, the headline stands
            r = {"error": f"{type(e).__name__}: {e}"}
        r["wall_s"] = time.perf_counter() - t0
        legs[name] = r
        torch.cuda.empty_cache()

    if "pressure" in want:
        leg("pressure", lambda: pressure_measure(dev, 2, 1))
    if "batch" in want:
        def batch():
            w = WORKLOADS["batch_512"]
            t0 = time.perf_counter()
            systems, _ = batch_systems(w["count"], w["seed"], w["tol"])
            t_gen = time.perf_counter() - t0
            m = batch_measure(systems, dev, 3, 1)
            m["generation_s"] = t_gen
            m["config"] = {"systems": w["count"], "sizes": "per axis U{16..96}", "tol": w["tol"], "itmax": w["itmax"]}
            return m
        leg("batch_512", batch)
    if "serving" in want:
        def serving():
            w = WORKLOADS["serve_poisson"]
            t0 = time.perf_counter()
            pool = serve_pool(w["pool"], w["seed"])
            t_gen = time.perf_counter() - t0
            m = serve_measure(pool, 10.0, w["budget"], fracs=(0.5,))
            m["generation_s"] = t_gen
            m["config"] = {"sizes": "per axis log-uniform on [24, 160]", "pressure_share": 0.2, "tol": [1e-6, 1e-8],
                           "hbm_budget_gb": w["budget"] / 1e9,
                           "note": "10 s runs (the serve_poisson workload runs the 60 s of the spec)"}
            del pool
            return m
        leg("serving", serving)
    return legs


def run_ours(args) -> None:
    import torch

    from mfix_b200 import leq

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    w = args.workload
    sys0 = make_system(w)
    n = sys0.n
    dev = torch.device("cuda", local)
    if args.line_lanes:
        leq.set_option("line_lanes", args.line_lanes)
    A0 = torch.from_numpy(sys0.a).to(dev)
    B0 = torch.from_numpy(sys0.b).to(dev)
    A = torch.empty_like(A0)
    B = torch.empty_like(B0)
    X = torch.zeros(n, dtype=torch.float64, device=dev)

    def solve_device(precision: int, time_kernels: bool = False):
        A.copy_(A0)
        B.copy_(B0)
        X.zero_()
        torch.cuda.synchronize()
        leq.set_option("time_kernels", 1 if time_kernels else 0)
        rc, res = leq.batch_solve([sys0], precision=precision, on_device=True,
                                  pointers=[(A.data_ptr(), B.data_ptr(), X.data_ptr())])
        if rc != 0 or res[0].ier != 0:
            raise RuntimeError(f"solve failed rc={rc} ier={res[0].ier if res else None}: {leq.last_error()}")
        st = leq.last_stats()
        return res[0], st

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        import torch.distributed as dist

        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.only != "all":
        for _ in range(max(args.steps, 1)):
            r, st = solve_device(0 if args.only == "fp64" else 1)
        print(f"{args.only}: iterations {r.iterations} outer {r.outer_steps} device_ms {st['device_ms']:.3f} "
              f"line_lanes {leq.autotune_table()}")
        return

    # ---- FP64 drop-in (device resident)
    for _ in range(args.warmup):
        solve_device(0)
    barrier()
    fp64_ms, fp64_launch = [], 0
    for _ in range(args.steps):
        r64, st = solve_device(0)
        fp64_ms.append(st["device_ms"])
        fp64_launch += st["kernel_launches"]
    barrier()
    x64 = X.clone()
    fp64_iters = r64.iterations

    # ---- mixed form (device resident), the iteration body replayed as a CUDA graph
    for _ in range(args.warmup):
        solve_device(1)
    barrier()
    sampler = ClockSampler(local)
    mixed_ms, launches = [], 0
    t_wall0 = time.perf_counter()
    with sampler:
        for _ in range(args.steps):
            rm, st = solve_device(1)
            mixed_ms.append(st["device_ms"])
            launches += st["kernel_launches"]
        barrier()
    wall = time.perf_counter() - t_wall0
    xm = X.clone()
    # one more mixed solve, outside the timed steps, with events around every
    # J-line launch (direct launches instead of graph replay) for the roofline
    r_tk, st = solve_device(1, time_kernels=True)
    jl_ms, jl_n = st["jline_ms"], st["jline_launches"]
    work_m = work_launches(r_tk.iterations, r_tk.outer_steps)
    kt_mixed = leq.last_kernel_times()
    r64_tk, st64 = solve_device(0, time_kernels=True)
    work_64 = work_launches(r64_tk.iterations, 0)
    kt_fp64 = leq.last_kernel_times()
    leq.set_option("time_kernels", 0)

    # accuracy of both forms on the scaled system (A, B hold the scaled copies)
    def true_rel(x):
        from mfix_b200 import leq as L

        y = torch.empty_like(x)
        L.leq_matvec(L.geom(sys0.imax2, sys0.jmax2, sys0.kmax2, sys0.do_k), A.data_ptr(), x.data_ptr(), y.data_ptr())
        r = B - y
        return float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(B))

    rel64, relm = true_rel(x64), true_rel(xm)
    diff = float(torch.linalg.vector_norm(xm - x64) / torch.linalg.vector_norm(x64))

    tot_mixed = max_over_ranks(sum(mixed_ms))
    tot_64 = max_over_ranks(sum(fp64_ms))
    value = world * args.steps / (tot_mixed / 1e3)
    fp64_value = world * args.steps / (tot_64 / 1e3)

    # ---- e2e through the Fortran-convention entry point, pinned host arrays:
    # the copies of A_M, B_M, VAR in and of VAR and the scaled A_M/B_M out are
    # inside the timing (mixed form: the headline; FP64 drop-in beside it)
    a_h = torch.empty((7, n), dtype=torch.float64).pin_memory().numpy()
    b_h = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    x_h = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    leq.init_geometry(sys0.imax2, sys0.jmax2, sys0.kmax2, 1, n, 0)

    def e2e(precision: int, steps: int, warm: int) -> float:
        leq.set_option("precision", precision)
        e2e_t = []
        for it in range(warm + steps):
            np.copyto(a_h, sys0.a)
            np.copyto(b_h, sys0.b)
            x_h[:] = 0.0
            barrier()
            t0 = time.perf_counter()
            ier = leq.solve_lin_eq("Pp_g", 1, x_h, a_h, b_h, 0, sys0.itmax, 2, "RSRS", sys0.tol, "LINE")
            t1 = time.perf_counter()
            if ier != 0:
                raise RuntimeError(f"e2e solve IER {ier}: {leq.last_error()}")
            if it >= warm:
                e2e_t.append(t1 - t0)
        leq.set_option("precision", 0)
        return world * steps / max_over_ranks(sum(e2e_t))

    e2e_value = e2e(1, args.steps, args.warmup)
    e2e_fp64_steps = max(3, args.steps // 2)
    e2e_fp64 = e2e(0, e2e_fp64_steps, 1)

    # ---- roofline of the J-line sweep kernel (FP32 in the mixed form)
    peak, peak_kind = measured_peak_hbm()
    alg_bytes_launch = 5 * 4 * n  # half the cells x (7 diagonals + rhs + guess + write) x 4 bytes
    jl_work = min(work_m["jline"], jl_n)  # launches that did work (the rest returned at once)
    avg_launch_s = (jl_ms / 1e3) / max(jl_work, 1)
    achieved = alg_bytes_launch / avg_launch_s / 1e9
    traffic = ncu_traffic(f"jline_f32_{w}.md")
    roof = {"kernel": "k_jline<float> (LINE preconditioner half-sweep)", "bound": "hbm", "achieved": achieved,
            "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": f"{peak_kind} (MEASURED_PEAKS hbm_gbs)",
            "alg_bytes_per_launch": alg_bytes_launch, "avg_launch_ms": avg_launch_s * 1e3, "launches": jl_n,
            "work_launches": jl_work, "traffic": traffic}

    # whole-solve algorithmic bandwidth
    mixed_bytes = n * (rm.iterations * BYTES_FP32_ITER + rm.outer_steps * BYTES_OUTER + BYTES_SETUP + 7 * 12)
    fp64_bytes = n * (fp64_iters * BYTES_FP64_ITER + BYTES_SETUP + 80)
    line = {
        "metric": "solves/s", "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot_mixed / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32-inner/fp64-refinement", "data": "synthetic",
        "config": workload_config(w, sys0),
        "roofline": roof,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": 9 * 8 * n,
                "d2h_bytes_per_step": 9 * 8 * n, "entry": "mfixgpu_solve_lin_eq_ (pinned host A_M/B_M/VAR)",
                "fp64_drop_in": {"value": e2e_fp64, "unit": "solves/s", "steps": e2e_fp64_steps,
                                 "h2d_bytes_per_step": 9 * 8 * n, "d2h_bytes_per_step": 9 * 8 * n}},
        "gpu_launches": int(launches),
        "clocks": sampler.summary(),
        "mixed": {"solves_per_s": value, "ms_per_solve": tot_mixed / args.steps, "inner_iterations": rm.iterations,
                  "outer_steps": rm.outer_steps, "true_rel_resid": relm, "alg_gbs": mixed_bytes / (tot_mixed / args.steps / 1e3) / 1e9,
                  "rel_diff_vs_fp64": diff},
        "fp64": {"solves_per_s": fp64_value, "ms_per_solve": tot_64 / args.steps, "iterations": fp64_iters,
                 "true_rel_resid": rel64, "alg_gbs": fp64_bytes / (tot_64 / args.steps / 1e3) / 1e9,
                 "gpu_launches": int(fp64_launch)},
        "mixed_vs_fp64": value / fp64_value,
        "line_tiles": [{"elem_bytes": e, "line_length": l, "lanes_per_line": g} for e, l, g in leq.autotune_table()],
        "kernels_mixed": class_table(kt_mixed, n, True, peak, work_m),
        "kernels_fp64": class_table(kt_fp64, n, False, peak, work_64),
        "wall_s_timed_mixed": wall,
    }
    if world == 1 and args.legs:
        # the other configurations (after the headline's own measurements)
        del A0, B0, A, B, X, a_h, b_h, x_h
        torch.cuda.empty_cache()
        line["legs"] = run_legs(args, dev)
    if rank == 0 and world == 1 and not args.no_cpu:
        import oracle as O

        # one complete oracle solve (the CPU baseline), then the accuracy of both
        # forms against the oracle's solution and against the 1e-14 truth
        t_cpu, ref, st_ref = cpu_solve(sys0)
        line["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
                                "sample": f"one complete oracle solve of the same system ({st_ref['iterations']} "
                                          f"iterations, {t_cpu:.1f} s)",
                                "gbs": BYTES_FP64_ITER * st_ref["iterations"] * n / t_cpu / 1e9}
        acc = accuracy(ref, st_ref, {"fp64": x64.cpu().numpy(), "mixed": xm.cpu().numpy()})
        line["accuracy"] = acc
        for form in ("fp64", "mixed"):
            line[form]["err_vs_truth"] = acc[form]["err_vs_truth"]
            line[form]["rel_diff_vs_oracle"] = acc[form]["rel_diff_vs_oracle"]
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


# Algorithmic bytes per cell of one FP64 CG iteration (model/leq_cg.f:271-410),
# fused minimum in words: MSOLVE 20 (two R letters: 2 reads of the 7 diagonals,
# 2 red/black passes of rhs + guess + write), matvec 9, rho 2, P 3, X/R 6.
BYTES_CG_ITER = 8 * (20 + 9 + 2 + 3 + 6)


def run_cg_bench(args) -> None:
    """METHOD 5 through the drop-in: device time of the solve with its inputs
    already on the device (setup + iterations, from the library's events), and
    end to end with pinned host arrays; the J-line kernel's roofline from a
    solve with events around every launch."""
    import torch

    from mfix_b200 import leq

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    w = args.workload
    sys0 = make_system(w)
    n = sys0.n
    dev = torch.device("cuda", local)
    a_h = torch.empty((7, n), dtype=torch.float64).pin_memory().numpy()
    b_h = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    x_h = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    leq.init_geometry(sys0.imax2, sys0.jmax2, sys0.kmax2, 1, n, 0)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        import torch.distributed as dist

        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def solve():
        np.copyto(a_h, sys0.a)
        np.copyto(b_h, sys0.b)
        x_h[:] = 0.0
        barrier()
        t0 = time.perf_counter()
        ier = leq.solve_lin_eq("Pp_g", 1, x_h, a_h, b_h, 0, sys0.itmax, 5, "RSRS", sys0.tol, "LINE")
        t1 = time.perf_counter()
        if ier != 0:
            raise RuntimeError(f"CG solve IER {ier}: {leq.last_error()}")
        return t1 - t0, leq.last_stats()

    for _ in range(args.warmup):
        solve()
    sampler = ClockSampler(local)
    walls, dev_ms, launches = [], [], 0
    with sampler:
        for _ in range(args.steps):
            wl, st = solve()
            walls.append(wl)
            dev_ms.append(st["device_ms"])
            launches += st["kernel_launches"]
        barrier()
    iters = st["iterations"]
    leq.set_option("time_kernels", 1)
    _, stk = solve()
    kt = leq.last_kernel_times()
    leq.set_option("time_kernels", 0)
    peak, peak_kind = measured_peak_hbm()
    tot_dev = max_over_ranks(sum(dev_ms))
    value = world * args.steps / (tot_dev / 1e3)
    e2e_value = world * args.steps / max_over_ranks(sum(walls))
    jl_ms, jl_n = stk["jline_ms"], stk["jline_launches"]
    its_tk = stk["iterations"]
    jl_work = min(4 * its_tk, jl_n)  # one MSOLVE (two R letters, four half-sweeps) per iteration
    alg_launch = 5 * 8 * n
    avg_s = (jl_ms / 1e3) / max(jl_work, 1)
    achieved = alg_launch / avg_s / 1e9
    rel = true_rel_resid(sys0, x_h, rows="diag")
    kernels = {}
    names = {"jline": "jline", "s_update": "cg_rho", "p_update": "cg_p", "matvec_alpha": "cg_matvec",
             "xr_update": "cg_xr"}
    cls_bytes = {"jline": 40, "s_update": 16, "p_update": 24, "matvec_alpha": 72, "xr_update": 48}
    for k, (ms, nl) in kt.items():
        if nl == 0 or k not in names:
            continue
        nw = min(jl_work if k == "jline" else its_tk, nl)  # launches after convergence return at once
        gbs = cls_bytes[k] * n * nw / (ms / 1e3) / 1e9
        kernels[names[k]] = {"ms": round(ms, 3), "launches": nl, "work_launches": nw,
                             "us_per_launch": round(1e3 * ms / max(nw, 1), 2), "gbs": round(gbs, 1),
                             "frac": round(gbs / peak, 3)}
    line = {
        "metric": "solves/s", "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot_dev / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w, "grid": list(WORKLOADS[w]["dims"]), "cells": n, "method": 5, "pc": "LINE",
                   "sweep": "RSRS", "tol": sys0.tol, "itmax": sys0.itmax,
                   "l2_policy": "inputs larger than L2 (A_M 7*8*cells bytes), no flush needed"},
        "roofline": {"kernel": "k_jline<double> (LINE preconditioner half-sweep)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "alg_bytes_per_launch": alg_launch, "avg_launch_ms": avg_s * 1e3,
                     "launches": jl_n, "work_launches": jl_work, "traffic": ncu_traffic(f"jline_f64_{w}.md")},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": 9 * 8 * n,
                "d2h_bytes_per_step": 9 * 8 * n, "entry": "mfixgpu_solve_lin_eq_ METHOD 5 (pinned host arrays)"},
        "gpu_launches": int(launches),
        "clocks": sampler.summary(),
        "iterations": iters, "true_rel_resid": rel,
        "alg_gbs": n * (iters * BYTES_CG_ITER + BYTES_SETUP + 80) / (tot_dev / args.steps / 1e3) / 1e9,
        "kernels": kernels,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        import oracle as O

        t = sys0.copy()
        t0 = time.perf_counter()
        st_ref = O.leq_cg(t)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
                                "sample": f"one complete oracle CG solve ({st_ref['iterations']} iterations)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def _alg_bytes(n: int, precision: int, iterations: int, outer: int, fallback_iters: int = 0) -> float:
    """Algorithmic bytes of one solve: per-iteration traffic of the fused minimum,
    FP64 refinement steps, setup (scaling + initial residual, FP32 copy of A)."""
    if precision == 1:
        return n * (iterations * BYTES_FP32_ITER + outer * BYTES_OUTER + BYTES_SETUP + 7 * 12 +
                    fallback_iters * BYTES_FP64_ITER)
    return n * (iterations * BYTES_FP64_ITER + BYTES_SETUP + 80)


def batch_measure(systems, dev, steps: int, warmup: int, barrier=None, mx=None, sm=None) -> dict:
    """The batched mixed form (every launch covers all systems) and the FP64 forms
    on the same device arrays: `steps` timed mixed batches after `warmup`, one
    FP64 batch, one loop of FP64 single-system solves.  mx / sm reduce a value
    over ranks (max / sum); the defaults are the identity (one rank)."""
    import torch

    from mfix_b200 import leq

    barrier = barrier or (lambda: torch.cuda.synchronize())
    mx = mx or (lambda v: v)
    sm = sm or (lambda v: v)
    pristine = [(torch.from_numpy(x.a).to(dev), torch.from_numpy(x.b).to(dev)) for x in systems]
    work = [(torch.empty_like(a), torch.empty_like(b), torch.zeros(x.n, dtype=torch.float64, device=dev))
            for (a, b), x in zip(pristine, systems)]
    ptrs = [(a.data_ptr(), b.data_ptr(), xx.data_ptr()) for a, b, xx in work]

    def reset():
        for (a0, b0), (a, b, xx) in zip(pristine, work):
            a.copy_(a0)
            b.copy_(b0)
            xx.zero_()
        torch.cuda.synchronize()

    def batched(precision):
        reset()
        t = time.perf_counter()
        rc, res = leq.batch_solve(systems, precision=precision, on_device=True, pointers=ptrs)
        wall = time.perf_counter() - t
        if rc != 0 or any(r.ier != 0 for r in res):
            raise RuntimeError(f"batch rc={rc} {leq.last_error()} iers={sorted(set(r.ier for r in res))}")
        st = leq.last_stats()
        return res, st["device_ms"] / 1e3, wall, st["kernel_launches"]

    def loop_fp64():
        reset()
        dev_s, res, launches = 0.0, [], 0
        t = time.perf_counter()
        for q, x in enumerate(systems):
            rc, r = leq.batch_solve([x], precision=0, on_device=True, pointers=[ptrs[q]])
            if rc != 0 or r[0].ier != 0:
                raise RuntimeError(f"single solve {q}: rc={rc} {leq.last_error()}")
            st = leq.last_stats()
            dev_s += st["device_ms"] / 1e3
            launches += st["kernel_launches"]
            res.append(r[0])
        return res, dev_s, time.perf_counter() - t, launches

    for _ in range(warmup):
        batched(1)
    batched(0)  # warm: each form's line shapes tuned on the whole batch (single solves tune one length alone)
    loop_fp64()  # warm: graph paths of the single solves
    barrier()
    mixed = [batched(1) for _ in range(steps)]
    barrier()
    fp64b = [batched(0) for _ in range(max(1, steps // 2))]
    loop = loop_fp64()
    barrier()
    peak, peak_kind = measured_peak_hbm()
    rm = mixed[-1][0]
    m_dev = mx(float(np.mean([m[1] for m in mixed])))
    m_wall = mx(float(np.mean([m[2] for m in mixed])))
    alg_m = sm(sum(_alg_bytes(x.n, 1, r.iterations, r.outer_steps) for x, r in zip(systems, rm)))
    alg_64 = sm(sum(_alg_bytes(x.n, 0, r.iterations, 0) for x, r in zip(systems, loop[0])))
    f_dev = mx(float(np.mean([m[1] for m in fp64b])))
    alg_f = sm(sum(_alg_bytes(x.n, 0, r.iterations, 0) for x, r in zip(systems, fp64b[-1][0])))
    loop_dev, loop_wall, loop_launch = mx(loop[1]), mx(loop[2]), int(sm(loop[3]))
    nsys = int(sm(len(systems)))
    return {
        "systems": nsys, "cells": int(sm(sum(x.n for x in systems))), "steps": steps,
        "mixed_batched": {"solves_per_s_device": nsys / m_dev, "solves_per_s_wall": nsys / m_wall,
                          "ms_per_batch": m_dev * 1e3, "alg_gbs": alg_m / m_dev / 1e9,
                          "frac_of_peak": alg_m / m_dev / 1e9 / peak, "peak_gbs": peak, "peak_kind": peak_kind,
                          "fp64_fallbacks": sum(r.fp64_fallback for r in rm), "gpu_launches": int(mixed[-1][3]),
                          "iterations_mean": float(np.mean([r.iterations for r in rm]))},
        "fp64_batched": {"solves_per_s_device": nsys / f_dev, "alg_gbs": alg_f / f_dev / 1e9,
                         "frac_of_peak": alg_f / f_dev / 1e9 / peak},
        "fp64_loop": {"solves_per_s_device": nsys / loop_dev, "solves_per_s_wall": nsys / loop_wall,
                      "alg_gbs": alg_64 / loop_dev / 1e9, "gpu_launches": loop_launch,
                      "iterations_mean": float(np.mean([r.iterations for r in loop[0]]))},
        "mixed_batched_vs_fp64_batched": f_dev / m_dev,
        "mixed_batched_vs_fp64_loop_device": loop_dev / m_dev,
        "mixed_batched_vs_fp64_loop_wall": loop_wall / m_wall,
    }


def batch_systems(count: int, seed: int, tol: float, indices=None):
    """The batch workload's systems (per-axis sizes U{16..96}), generated in spawned
    processes; `indices` selects a subset (a rank's share)."""
    from mfix_b200 import systems as S

    sizes = S.batch_sizes(count, seed)
    specs = [("conv_diff", d, tol, q) for q, d in enumerate(sizes)]
    if indices is not None:
        specs = [specs[q] for q in indices]
    return generate_systems(specs), sizes


def run_batch_bench(args) -> None:
    """512 uneven systems: one batched mixed-precision solve (every launch covers
    all systems) vs a loop of plain FP64 single-system solves on the same arrays."""
    import torch

    from mfix_b200 import leq
    from mfix_b200 import shard
    from mfix_b200 import systems as S

    rank, world, local = dist_env()
    w = WORKLOADS[args.workload]
    sizes = S.batch_sizes(w["count"], w["seed"])
    # ranks share the independent systems (no collective on the data path)
    mine = shard.assign([(i + 2) * (j + 2) * (k + 2) for i, j, k in sizes], world)[rank]
    t0 = time.perf_counter()
    systems, _ = batch_systems(w["count"], w["seed"], w["tol"], mine)
    t_gen = time.perf_counter() - t0
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    if args.only != "all":  # profiling runs: the batched solve of one form only
        if args.line_lanes:
            leq.set_option("line_lanes", args.line_lanes)
        import torch as _t

        pristine = [(_t.from_numpy(x.a).to(dev), _t.from_numpy(x.b).to(dev)) for x in systems]
        ptrs = []
        work = []
        for (a0, b0), x in zip(pristine, systems):
            a, b, xx = a0.clone(), b0.clone(), _t.zeros(x.n, dtype=_t.float64, device=dev)
            work.append((a, b, xx))
            ptrs.append((a.data_ptr(), b.data_ptr(), xx.data_ptr()))

        def once(tk):
            for (a0, b0), (a, b, xx) in zip(pristine, work):
                a.copy_(a0)
                b.copy_(b0)
                xx.zero_()
            _t.cuda.synchronize()
            leq.set_option("time_kernels", tk)
            rc, res = leq.batch_solve(systems, precision=1 if args.only == "mixed" else 0, on_device=True,
                                      pointers=ptrs)
            leq.set_option("time_kernels", 0)
            if rc != 0:
                raise RuntimeError(leq.last_error())
            return res, leq.last_stats()

        for _ in range(args.warmup + args.steps):
            res, st = once(0)
        print(f"{args.only} batch: {len(systems)} systems, {st['device_ms']:.1f} ms, {st['kernel_launches']} launches, "
              f"iterations max {max(r.iterations for r in res)} mean {np.mean([r.iterations for r in res]):.1f}")
        res, st = once(1)
        print(f"  timed J-line launches: {st['jline_launches']} in {st['jline_ms']:.1f} ms of {st['device_ms']:.1f} ms; "
              f"lanes {sorted(set(g for e, l, g in leq.autotune_table()))}")
        for k, (ms, nl) in leq.last_kernel_times().items():
            print(f"  {k:14s} {ms:9.2f} ms {nl:6d} launches")
        return
    sampler = ClockSampler(local)
    with sampler:
        m = batch_measure(systems, dev, args.steps, args.warmup, barrier,
                          lambda v: shard.max_over_ranks(v, dev), lambda v: shard.sum_over_ranks(v, dev))
    mb = m["mixed_batched"]
    peak, peak_kind = measured_peak_hbm()
    line = {
        "metric": "solves/s", "value": mb["solves_per_s_device"], "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": mb["ms_per_batch"], "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "fp32-inner/fp64-refinement", "data": "synthetic",
        "config": {"workload": args.workload, "systems": m["systems"], "cells": m["cells"],
                   "sizes": "per axis U{16..96}", "parallelism": f"systems sharded over {world} rank(s), longest first",
                   "pc": "LINE", "sweep": "RSRS", "tol": w["tol"], "itmax": w["itmax"],
                   "l2_policy": "inputs larger than L2 (A_M of the batch 7*8*cells bytes)"},
        "roofline": {"kernel": "whole batched solve (algorithmic bytes)", "bound": "hbm", "achieved": mb["alg_gbs"],
                     "peak": peak, "unit": "GB/s", "frac": mb["frac_of_peak"], "peak_kind": peak_kind, "traffic": None},
        "e2e": None,
        "gpu_launches": mb["gpu_launches"],
        "clocks": sampler.summary(),
        "generation_s": t_gen,
        **{k: v for k, v in m.items() if k not in ("systems", "cells", "steps")},
    }
    if not args.no_cpu and rank == 0 and world == 1:
        import oracle as O

        t = time.perf_counter()
        k = 0
        while k < len(systems) and (k < 4 or time.perf_counter() - t < 15.0):
            c = systems[k].copy()
            O.leq_bicgs(c)
            k += 1
        dt = time.perf_counter() - t
        line["cpu_baseline"] = {"value": k / dt, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
                                "sample": f"the first {k} of the {len(systems)} systems solved completely"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


class _Req:
    """A request: a pool system's arrays with the request's TOL."""
    __slots__ = ("imax2", "jmax2", "kmax2", "do_k", "n", "a", "b", "x", "tol", "itmax")

    def __init__(self, s, x, tol):
        self.imax2, self.jmax2, self.kmax2, self.do_k = s.imax2, s.jmax2, s.kmax2, s.do_k
        self.n, self.a, self.b, self.x, self.tol, self.itmax = s.n, s.a, s.b, x, tol, s.itmax


def _serve_run(leq, pool, precision, rate, seconds, seed, budget, check_every=8, max_systems=512,
               verify_every=40):
    check_every = SERVE_CHECK_EVERY or check_every
    """One open-loop Poisson run against a fresh server; returns its statistics."""
    rng = np.random.default_rng(seed)
    nreq = int(rate * seconds * 1.2) + 16
    arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
    arrivals = arrivals[arrivals < seconds]
    # requests walk the pool of distinct systems in order (from a random start), so
    # no system repeats before the pool is exhausted; each keeps its own TOL
    which = (int(rng.integers(0, len(pool))) + np.arange(len(arrivals))) % len(pool)
    tols = np.array([pool[q].tol for q in which])
    shared_x = [np.empty(p.n) for p in pool]  # outputs of unverified requests (never read)
    results, private = {}, {}
    srv = leq.Server(precision=precision, max_systems=max_systems, check_every=check_every, hbm_budget=budget)
    # warm the live batches (graph capture paths, memory pool)
    warm = [srv.submit(_Req(pool[q], np.empty(pool[q].n), 1e-6), zero_guess=True) for q in range(min(16, len(pool)))]
    for t in warm:
        srv.wait(t, 600)
    done_evt = threading.Event()

    def collector():
        while not (done_evt.is_set() and len(results) >= submitted[0]):
            got = srv.wait_any(0.2)
            if got is not None:
                results[got[0]] = got[1]

    submitted = [0]
    tickets = {}
    th = threading.Thread(target=collector, daemon=True)
    th.start()
    c0 = srv.counters()
    t_start = time.perf_counter()
    srv_t0 = c0["seconds"]
    for i, (ta, q) in enumerate(zip(arrivals, which)):
        delay = t_start + ta - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        if verify_every and i % verify_every == 0:
            x = np.empty(pool[q].n)
            private[i] = (q, x)
        else:
            x = shared_x[q]
        t = srv.submit(_Req(pool[q], x, float(tols[i])), zero_guess=True)
        if t < 0:
            raise RuntimeError(f"submit failed: {t} {leq.last_error()}")
        tickets[t] = i
        submitted[0] += 1
    window_end = srv_t0 + seconds
    while time.perf_counter() < t_start + seconds:
        time.sleep(0.01)
    c_end = srv.counters()
    srv.cancel_queued()
    done_evt.set()
    th.join(timeout=900)
    c_fin = srv.counters()
    srv.close()
    recs = [(tickets[t], r) for t, r in results.items()]
    ok = [(i, r) for i, r in recs if r["ier"] != leq.IER_CANCELLED]
    cancelled = sum(1 for _, r in recs if r["ier"] == leq.IER_CANCELLED)
    in_window = [(i, r) for i, r in ok if r["t_done"] <= window_end]
    lat = np.array([r["t_done"] - r["t_submit"] for _, r in ok]) * 1e3
    queue = np.array([r["t_admit"] - r["t_submit"] for _, r in ok]) * 1e3
    alg = sum(_alg_bytes(pool[which[i]].n, precision, r["mixed_iterations"] if r["fp64_fallback"] else r["iterations"],
                         r["outer_steps"], r["iterations"] if r["fp64_fallback"] else 0) for i, r in in_window)
    bad = [r["ier"] for _, r in ok if r["ier"] != 0]
    pct = (lambda a, p: float(np.percentile(a, p)) if len(a) else None)
    return {
        "precision": "mixed" if precision == 1 else "fp64", "offered_rate": rate, "seconds": seconds,
        "submitted": len(arrivals), "completed": len(ok), "completed_in_window": len(in_window),
        "served_rate": len(in_window) / seconds, "cancelled_backlog": cancelled,
        "backlog_at_window_end": int(c_end["queued"] + c_end["copying"]),
        "latency_ms": {"p50": pct(lat, 50), "p99": pct(lat, 99), "mean": float(lat.mean()) if len(lat) else None},
        "queue_wait_ms": {"p50": pct(queue, 50), "p99": pct(queue, 99)},
        "alg_gbs": alg / seconds / 1e9, "fp64_fallbacks": int(c_fin["fp64_fallbacks"]),
        "max_running": int(c_fin["max_running"]), "peak_reserved_gb": c_fin["peak_reserved_bytes"] / 1e9,
        "budget_gb": c_fin["budget_bytes"] / 1e9, "commits": int(c_fin["commits"] - c0["commits"]),
        "iteration_bodies": int(c_fin["iterations"] - c0["iterations"]),
        "gpu_launches": int(c_fin["kernel_launches"] - c0["kernel_launches"]),
        "nonzero_ier": len(bad), "_private": private, "_results": {tickets[t]: r for t, r in results.items()},
        "_tols": tols,
    }


SERVE_CHECK_EVERY = 0  # --serve-check: iterations between state reads in the serving runs (0: 8)


def _serve_closed(leq, pool, precision, inflight, seconds, seed, budget, check_every=8, max_systems=512):
    check_every = SERVE_CHECK_EVERY or check_every
    """Closed loop: `inflight` requests outstanding, each completion replaced by a
    new request, for `seconds`; the completion rate is the server's capacity for
    the request mix (completions follow the submission mix in steady state)."""
    rng = np.random.default_rng(seed)
    xs = [np.empty(p.n) for p in pool]  # outputs (never read)
    srv = leq.Server(precision=precision, max_systems=max_systems, check_every=check_every, hbm_budget=budget)
    which = {}
    nxt = [int(rng.integers(0, len(pool)))]  # requests walk the pool of distinct systems in order

    def submit():
        q = nxt[0] % len(pool)
        nxt[0] += 1
        t = srv.submit(_Req(pool[q], xs[q], pool[q].tol), zero_guess=True)
        if t < 0:
            raise RuntimeError(f"submit failed: {t} {leq.last_error()}")
        which[t] = q
        return t

    for _ in range(min(16, inflight)):  # warm the live batches
        t = submit()
        srv.wait(t, 600)
        which.pop(t)
    c0 = srv.counters()
    t_end = c0["seconds"] + seconds
    warm_until = c0["seconds"] + 0.2 * seconds
    for _ in range(inflight):
        submit()
    done = []
    stall = 0
    while True:
        got = srv.wait_any(5.0)
        if got is None:
            stall += 1
            if stall > 120:  # ten minutes without a completion
                raise RuntimeError("serving run made no progress")
            continue
        stall = 0
        t, r = got
        done.append((which.pop(t), r))
        if r["t_done"] < t_end:
            submit()
        elif not which:
            break
    c1 = srv.counters()
    srv.close()
    win = [(q, r) for q, r in done if warm_until <= r["t_done"] < t_end]
    span = t_end - warm_until
    alg = sum(_alg_bytes(pool[q].n, precision, r["mixed_iterations"] if r["fp64_fallback"] else r["iterations"],
                         r["outer_steps"], r["iterations"] if r["fp64_fallback"] else 0) for q, r in win)
    lat = np.array([r["t_done"] - r["t_submit"] for _, r in win]) * 1e3
    return {"precision": "mixed" if precision == 1 else "fp64", "inflight": inflight, "seconds": seconds,
            "window_s": span, "completed_in_window": len(win), "capacity": len(win) / span,
            "alg_gbs": alg / span / 1e9, "latency_ms_at_capacity": {"p50": float(np.percentile(lat, 50)),
                                                                    "p99": float(np.percentile(lat, 99))},
            "fp64_handovers": int(c1["fp64_fallbacks"] - c0["fp64_fallbacks"]),
            "device_busy_frac": [round((c1["busy_ms"][k] - c0["busy_ms"][k]) / (1e3 * (c1["seconds"] - c0["seconds"])), 3)
                                 for k in range(2)],
            "nonzero_ier": sum(1 for _, r in done if r["ier"] != 0)}


def serve_pool(count: int, seed: int):
    """The serving workload's pool of distinct request systems (per-axis sizes
    log-uniform on [24, 160], 20% pressure-like, TOL from {1e-6, 1e-8}), generated
    in spawned processes, with pinned host copies of A_M and B_M (the server's
    copies overlap the iterations)."""
    import torch

    from mfix_b200 import systems as S

    pool = generate_systems(S.serve_mix(count, seed))
    for p in pool:
        a = torch.empty(p.a.shape, dtype=torch.float64).pin_memory().numpy()
        b = torch.empty(p.b.shape, dtype=torch.float64).pin_memory().numpy()
        np.copyto(a, p.a)
        np.copyto(b, p.b)
        p.a, p.b = a, b
    return pool


def serve_measure(pool, seconds: float, budget: float, fracs=(0.5,), offered=None) -> dict:
    """Capacity of both forms from closed-loop runs (256 requests in flight), p50/p99
    latency of both forms from Poisson streams at `fracs` of the FP64 capacity (the
    same offered load for both), optionally the stream at `offered` req/s
    (saturating: served rate and backlog); a sample of results checked against the
    FP64 true residual."""
    from mfix_b200 import leq

    peak, peak_kind = measured_peak_hbm()
    cap_m = _serve_closed(leq, pool, 1, 256, seconds, 11, budget)
    cap_f = _serve_closed(leq, pool, 0, 256, seconds, 11, budget)
    loads = []
    for frac in fracs:
        lam = frac * cap_f["capacity"]
        loads.append((frac, _serve_run(leq, pool, 1, lam, seconds, 2, budget),
                      _serve_run(leq, pool, 0, lam, seconds, 2, budget)))
    sat = _serve_run(leq, pool, 1, offered, min(seconds, 10.0), 1, budget) if offered else None
    worst, checked = 0.0, 0
    for _, rm, rf in loads:
        for r in (rm, rf):
            for i, (q, x) in list(r["_private"].items())[:6]:
                res = r["_results"].get(i)
                if res is None or res["ier"] != 0:
                    continue
                rel = true_rel_resid(pool[q], x)
                worst = max(worst, rel / float(r["_tols"][i]))
                checked += 1
    strip = lambda r: {k: v for k, v in r.items() if not k.startswith("_")}
    half = loads[0]
    out = {
        "pool_systems": len(pool), "pool_cells_mean": float(np.mean([p.n for p in pool])), "seconds_per_run": seconds,
        "capacity": {"mixed": cap_m, "fp64": cap_f, "mixed_vs_fp64": cap_m["capacity"] / cap_f["capacity"]},
        "capacity_frac_of_peak": {"mixed": cap_m["alg_gbs"] / peak, "fp64": cap_f["alg_gbs"] / peak,
                                  "peak_gbs": peak, "peak_kind": peak_kind},
        "latency": {f"{int(100 * frac)}pct_of_fp64_capacity": {"offered_rate": rm["offered_rate"], "mixed": strip(rm),
                                                               "fp64": strip(rf)} for frac, rm, rf in loads},
        "p50_p99_ms": {"mixed": [half[1]["latency_ms"]["p50"], half[1]["latency_ms"]["p99"]],
                       "fp64": [half[2]["latency_ms"]["p50"], half[2]["latency_ms"]["p99"]],
                       "offered_rate": half[1]["offered_rate"]},
        "verified_requests": checked, "worst_true_resid_over_tol": worst,
        "gpu_launches": half[1]["gpu_launches"],
    }
    if sat is not None:
        out["offered_stream"] = strip(sat)
    return out


def run_serve_bench(args) -> None:
    """The request server on a stream of mixed-size requests, mixed form vs FP64
    form: capacity from closed-loop runs, p50/p99 latency from Poisson streams at
    50% and 80% of the FP64 capacity (the same offered load for both forms), and
    the workload's own offered rate (saturating) with served rate and backlog."""
    import torch

    w = WORKLOADS[args.workload]
    rate = args.rate or w["rate"]
    seconds = args.seconds or w["seconds"]
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    pool = serve_pool(w["pool"], w["seed"])
    t_gen = time.perf_counter() - t0
    sampler = ClockSampler(0)
    with sampler:
        m = serve_measure(pool, seconds, w["budget"], fracs=(0.5, 0.8), offered=rate)
    peak, peak_kind = measured_peak_hbm()
    cap_m = m["capacity"]["mixed"]
    line = {
        "metric": "solves/s & p50/p99 latency", "value": cap_m["capacity"], "unit": "solves/s", "n_gpus": 1,
        "steps": 1, "warmup": 1, "ms_per_step": seconds * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32-inner/fp64-refinement", "data": "synthetic",
        "config": {"workload": args.workload, "seconds_per_run": seconds, "pool_systems": len(pool),
                   "pool_cells_mean": m["pool_cells_mean"],
                   "sizes": "per axis log-uniform on [24, 160]", "pressure_share": 0.2, "tol": [1e-6, 1e-8],
                   "hbm_budget_gb": w["budget"] / 1e9, "max_systems_per_batch": 512,
                   "check_every": SERVE_CHECK_EVERY or 8,
                   "capacity": "closed loop, 256 requests in flight, completions after the first 20% of the run",
                   "inputs": "pinned host A_M/B_M copied in per request, VAR copied out; zero initial guess; "
                             "requests walk a pool of distinct systems"},
        "roofline": {"kernel": "served solves at capacity (algorithmic bytes of completed requests)", "bound": "hbm",
                     "achieved": cap_m["alg_gbs"], "peak": peak, "unit": "GB/s", "frac": cap_m["alg_gbs"] / peak,
                     "peak_kind": peak_kind, "traffic": None},
        "e2e": {"value": cap_m["capacity"], "unit": "solves/s", "note": "host arrays in and out per request"},
        "gpu_launches": m["gpu_launches"],
        "clocks": sampler.summary(),
        "generation_s": t_gen,
        **{k: v for k, v in m.items() if k not in ("gpu_launches",)},
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--legs", default="pressure,batch,serving",
                    help="default workload: the other configurations measured in the same run (comma list of "
                         "pressure, batch, serving; empty: none)")
    ap.add_argument("--line-lanes", type=int, default=0, help="force lanes per J-line (0: autotuned)")
    ap.add_argument("--rate", type=float, default=0.0, help="serving: offered requests/s (0: the workload's)")
    ap.add_argument("--serve-check", type=int, default=0, help="serving: iterations between state reads")
    ap.add_argument("--tune-cache", default="", help="JSON file of J-line lanes choices: loaded, and new choices "
                    "saved (a profiling run reuses the shapes of the timed run instead of tuning under the profiler)")
    ap.add_argument("--capacity-only", action="store_true", help="serving: the closed-loop capacity runs only")
    ap.add_argument("--seconds", type=float, default=0.0, help="serving: arrival window (0: the workload's)")
    ap.add_argument("--only", default="all", choices=["all", "fp64", "mixed"],
                    help="profiling runs: solve only this form (no e2e leg, no JSON line)")
    args = ap.parse_args()
    global SERVE_CHECK_EVERY
    SERVE_CHECK_EVERY = args.serve_check
    if args.tune_cache and args.impl != "reference":
        from mfix_b200 import leq

        leq.autotune_cache(args.tune_cache)
    kind = WORKLOADS[args.workload]["kind"]
    if args.impl == "reference":
        run_reference(args)
    elif kind == "batch":
        run_batch_bench(args)
    elif kind == "serve":
        run_serve_bench(args)
    elif kind == "cg":
        run_cg_bench(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
