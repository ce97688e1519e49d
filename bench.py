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
* cpu_baseline  the oracle (a C restatement of the reference's FP64 LEQ_BICGS with the
             reference's OpenMP loops) on a bounded sample of the same system.

``--impl reference`` times that CPU implementation alone (rank 0), with all host cores.
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
}
DEFAULT_WORKLOAD = "conv_diff_256"
# Iterations the reference FP64 algorithm needs on each seeded workload (the GPU FP64
# drop-in follows the same algorithm; tests/test_gpu_bench_workload.py checks it).
# Used by the CPU arm to turn a timed sample of iterations into solves/s.
FP64_ITERATIONS = {"conv_diff_256": 66, "conv_diff_64": 65, "conv_diff_192": None, "pressure_192x384x192": None}

BYTES_FP64_ITER = 576  # algorithmic bytes per cell per BiCGSTAB iteration, FP64 (72 words)
BYTES_FP32_ITER = 288  # the same in the FP32 inner solve
BYTES_OUTER = 104      # FP64 refinement step: r = b - A x (80) + x update (24)
BYTES_SETUP = 128      # unit scaling (16 w) of FP64 A and B


def make_system(name: str):
    from mfix_b200 import systems as S

    w = WORKLOADS[name]
    i, j, k = w["dims"]
    if w["kind"] == "conv_diff":
        return S.conv_diff(i, j, k, seed=w["seed"], itmax=w["itmax"], tol=w["tol"])
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


def cpu_sample(sys0, iters_needed: int | None, sample_iters=(2, 5)) -> dict:
    """Time the oracle (reference FP64 LEQ_BICGS restated in C, OpenMP) on a bounded
    sample: two runs of m1 and m2 iterations give the per-iteration time and the
    setup time; solves/s = 1 / (setup + iterations_needed * per_iteration)."""
    import oracle as O

    times = []
    for m in sample_iters:
        s = sys0.copy()
        t0 = time.perf_counter()
        O.leq_bicgs(s, max_exec=m)
        times.append(time.perf_counter() - t0)
    m1, m2 = sample_iters
    t_iter = max((times[1] - times[0]) / (m2 - m1), 1e-9)
    t_setup = max(times[0] - m1 * t_iter, 0.0)
    n = sys0.n
    out = {"cores": O.num_threads(), "kind": "port", "t_iter_s": t_iter, "t_setup_s": t_setup,
           "sample": f"{m1} and {m2} BiCGSTAB iterations of the {sys0.imax2}x{sys0.jmax2}x{sys0.kmax2}-cell system "
                     f"(setup + per-iteration time), scaled to the {iters_needed} iterations a full FP64 solve takes",
           "gbs": BYTES_FP64_ITER * n / t_iter / 1e9}
    if iters_needed:
        t_solve = t_setup + iters_needed * t_iter
        out["value"] = 1.0 / t_solve
        out["unit"] = "solves/s"
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
    sys0 = make_system(w)
    iters = FP64_ITERATIONS.get(w)
    vals = []
    for _ in range(args.warmup):
        cpu_sample(sys0, iters)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_sample(sys0, iters))
    wall = time.perf_counter() - t0
    v = float(np.mean([x.get("value", float("nan")) for x in vals]))
    line = {"impl": "reference", "metric": "solves/s", "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v if v > 0 else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(w, sys0),
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": vals[0]["cores"], "kind": "port",
                             "sample": vals[0]["sample"]},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall, "cpu_gbs": float(np.mean([x["gbs"] for x in vals]))}
    print(json.dumps(line), flush=True)


def workload_config(w: str, s) -> dict:
    return {"workload": w, "grid": list(WORKLOADS[w]["dims"]), "cells": s.n, "pc": "LINE", "sweep": "RSRS",
            "tol": WORKLOADS[w]["tol"], "itmax": WORKLOADS[w]["itmax"], "batch": 1,
            "l2_policy": "inputs larger than L2 (A_M 7*8*cells bytes), no flush needed"}


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

    # ---- mixed form (device resident), J-line launches timed with events
    for _ in range(args.warmup):
        solve_device(1)
    barrier()
    sampler = ClockSampler(local)
    mixed_ms, jl_ms, jl_n, launches = [], 0.0, 0, 0
    t_wall0 = time.perf_counter()
    with sampler:
        for _ in range(args.steps):
            rm, st = solve_device(1, time_kernels=True)
            mixed_ms.append(st["device_ms"])
            jl_ms += st["jline_ms"]
            jl_n += st["jline_launches"]
            launches += st["kernel_launches"]
        barrier()
    wall = time.perf_counter() - t_wall0
    leq.set_option("time_kernels", 0)
    xm = X.clone()

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

    # ---- e2e through the Fortran-convention entry point, pinned host arrays
    a_h = torch.empty((7, n), dtype=torch.float64).pin_memory().numpy()
    b_h = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    x_h = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    leq.set_option("precision", 1)
    leq.init_geometry(sys0.imax2, sys0.jmax2, sys0.kmax2, 1, n, 0)
    e2e_t = []
    for it in range(args.warmup + args.steps):
        np.copyto(a_h, sys0.a)
        np.copyto(b_h, sys0.b)
        x_h[:] = 0.0
        barrier()
        t0 = time.perf_counter()
        ier = leq.solve_lin_eq("Pp_g", 1, x_h, a_h, b_h, 0, sys0.itmax, 2, "RSRS", sys0.tol, "LINE")
        t1 = time.perf_counter()
        if ier != 0:
            raise RuntimeError(f"e2e solve IER {ier}: {leq.last_error()}")
        if it >= args.warmup:
            e2e_t.append(t1 - t0)
    leq.set_option("precision", 0)
    e2e_tot = max_over_ranks(sum(e2e_t))
    e2e_value = world * args.steps / e2e_tot

    # ---- roofline of the J-line sweep kernel (FP32 in the mixed form)
    peak, peak_kind = measured_peak_hbm()
    alg_bytes_launch = 5 * 4 * n  # half the cells x (7 diagonals + rhs + guess + write) x 4 bytes
    avg_launch_s = (jl_ms / 1e3) / max(jl_n, 1)
    achieved = alg_bytes_launch / avg_launch_s / 1e9
    traffic = ncu_traffic(f"jline_f32_{w}.md")
    roof = {"kernel": "k_jline<float> (LINE preconditioner half-sweep)", "bound": "hbm", "achieved": achieved,
            "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": f"{peak_kind} (MEASURED_PEAKS hbm_gbs)",
            "alg_bytes_per_launch": alg_bytes_launch, "avg_launch_ms": avg_launch_s * 1e3, "launches": jl_n,
            "traffic": traffic}

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
                "d2h_bytes_per_step": 9 * 8 * n, "entry": "mfixgpu_solve_lin_eq_ (pinned host A_M/B_M/VAR)"},
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
        "wall_s_timed_mixed": wall,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_sample(sys0, fp64_iters)
        line["cpu_baseline"] = {"value": cb.get("value"), "unit": "solves/s", "cores": cb["cores"], "kind": "port",
                                "sample": cb["sample"], "gbs": cb["gbs"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--line-lanes", type=int, default=0, help="force lanes per J-line (0: autotuned)")
    ap.add_argument("--only", default="all", choices=["all", "fp64", "mixed"],
                    help="profiling runs: solve only this form (no e2e leg, no JSON line)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
