#!/usr/bin/env python3
"""Benchmark of the steady SIMPLE hot path on one B200 (one process per GPU).

Workload (named by the benchmark's metric): the ~1M-tet straight pipe,
O-grid 24 rings x 72 sectors (+ an 18x18 square core) x 100 slabs, 6 tets per
quad and slab = 1,231,200 tets, seed-1 jitter of +-5 % local spacing, Re = 100,
alpha_u 0.7, alpha_p 0.3, pressure PCG rtol 1e-6 with the smoothed-aggregation
AMG + Chebyshev(2) V-cycle.  Precision: amg_fp32 (FP64 state, momentum,
operator and Krylov method; FP32 V-cycle) by default, --precision fp64 for the
plain path.

Metric: seconds to steady state (relCont <= 1e-6 and the pre-sweep momentum
audit <= 1e-6).  A complete solve takes 4193 SIMPLE iterations and 75k
pressure PCG iterations, so a benchmark "step" is one SIMPLE outer iteration
(assembly, momentum sweep, continuity, fine Schur refresh, AMG-PCG pressure
solve, pressure update) and the timed steps calibrate

    value = N_outer x t_outer + N_pcg x t_pcg

where t_outer is the mean device time of a step outside its PCG iterations,
t_pcg the device time per PCG iteration (pressure-solve time / iterations
over the timed steps), and N_outer, N_pcg the outer and PCG iteration counts
of a complete solve of this exact configuration by this solver (the CPU
oracle follows the same iteration history, see tests/), recorded in
profiles/steady_state_pipe1m.md beside the measured complete-solve times.
The per-iteration working set (fine operator ~1 GB) is larger than the 126 MB
L2, so no flush is inserted.

Modes:
  python bench.py [--gpus N --steps K --warmup W]     this package (CUDA path)
  python bench.py --impl reference [...]                the CPU restatement of
      the reference's SIMPLE loop (oracle/, FP64, all host threads), same
      metric, workload and projection, each step one SIMPLE iteration
      (bounded sample).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "s to steady state (resid 1e-6): FP32+learned vs plain FP64 AMG-FGMRES, 1 B200"
WORKLOAD = "pipe1m"
OPTIONS = dict(re=100.0, alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, run_mode="converge", simple_tol=1e-6,
               max_outer=100000, amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg")
# Complete solves of OPTIONS on WORKLOAD to relCont <= 1e-6 plus the momentum
# audit (profiles/steady_state_pipe1m.md): outer and total PCG iterations.
STEADY_STATE = {"fp64": {"outer": 4193, "pcg": 75316}, "amg_fp32": {"outer": 4193, "pcg": 75402}}
STEADY_STATE_SOURCE = "profiles/steady_state_pipe1m.md"
PRECISION_NOTE = {"fp64": "FP64 throughout (the reference's FP64 build)",
                  "amg_fp32": "FP64 state, momentum, fine operator and PCG; FP32 AMG V-cycle"}


def project(outer_ms, pcg_ms, pcg_its, prec):
    """Seconds to steady state from per-step times outside PCG (outer_ms),
    per-step PCG times (pcg_ms) and per-step PCG iteration counts."""
    ss = STEADY_STATE[prec]
    t_outer = float(np.mean(outer_ms))
    t_pcg = float(np.sum(pcg_ms)) / max(int(np.sum(pcg_its)), 1)
    return (ss["outer"] * t_outer + ss["pcg"] * t_pcg) / 1e3, t_outer, t_pcg


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic():
    p = ROOT / "profiles" / "fine_spmv_traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("bytes_per_launch_pipe1m_fp64")
    return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _barrier_max(x: float, ws: int, device: int) -> float:
    """Max of x over the replicas (also the barrier around the timed region)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = f"cuda:{device}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def fine_spmv_bytes(problem, s: int) -> float:
    """Compulsory bytes of one fine Schur SpMV: values + columns + row offsets + x + y."""
    row = problem.array("fine.row")
    n = len(row) - 1
    nnz = int(row[-1])
    return nnz * (s + 4) + 4 * (n + 1) + 2 * s * n


def sell_format_bytes(problem, s: int) -> float:
    """Bytes the SELL-32x4 fine operator actually streams per SpMV: padded
    values (s B) and 16-bit column deltas (slice width rounded up to a
    multiple of 4), slice offsets/widths, x and y."""
    row = problem.array("fine.row")
    n = len(row) - 1
    lens = np.diff(row)
    ns = (n + 31) // 32
    w = np.zeros(ns * 32, dtype=np.int64)
    w[:n] = lens
    widths = (w.reshape(ns, 32).max(axis=1) + 3) // 4 * 4
    padded = int(widths.sum()) * 32
    return padded * (s + 2) + 8 * ns + 2 * s * n


def run_nodals(args):
    from nodals_b200 import meshgen
    from nodals_b200 import native as N
    ws, rank, local = _dist()
    if ws > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    prec = args.precision
    tm = meshgen.named(WORKLOAD)
    mesh = N.Mesh.from_tetmesh(tm)
    t0 = time.perf_counter()
    P = N.Problem(mesh, precision=prec, device=local, **OPTIONS)
    setup_s = time.perf_counter() - t0
    S = N.Solver(P)
    for _ in range(args.warmup):
        S.step()
    l0 = N.launch_count()
    _barrier_max(0.0, ws, local)
    with Clocks(local) as clk:
        dev_ms, outer_ms, pcg_ms, pcg_its = [], [], [], []
        w0 = time.perf_counter()
        for _ in range(args.steps):
            r = S.step()
            total = r.ms_assembly + r.ms_momentum + r.ms_continuity + r.ms_pressure + r.ms_update
            solve = r.ms_pressure - r.ms_refresh
            dev_ms.append(total)
            outer_ms.append(total - solve)
            pcg_ms.append(solve)
            pcg_its.append(r.p_its)
        wall = time.perf_counter() - w0
    launches = N.launch_count() - l0
    # Per-kernel CUDA events need the launch-by-launch path of the Krylov
    # loop, so the roofline kernel is timed in a profiled pass of further
    # steps of the same solve right after the timed region.
    S.profile(True)
    for _ in range(args.profile_steps):
        S.step()
    prof = S.profile_read()
    S.profile(False)
    mean_ms = float(np.mean(dev_ms))
    value, t_outer, t_pcg = project(outer_ms, pcg_ms, pcg_its, prec)
    if WORKLOAD != "pipe1m":
        value = 0.0  # the steady-state counts belong to pipe1m; smaller pipes serve profiling only
    value = _barrier_max(value, ws, local)
    mean_ms = _barrier_max(mean_ms, ws, local)
    calls, tot = prof["fine_spmv"]
    roof = None
    if args.profile_steps > 0:
        if calls == 0:
            raise RuntimeError("no fine SpMV launch was timed in the profiled pass")
        avg_launch_ms = tot / calls
        alg = fine_spmv_bytes(P, 8)
        fmt = sell_format_bytes(P, 8)
        peak, peak_kind = _peaks()
        achieved = alg / (avg_launch_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": _traffic(), "peak_kind": peak_kind,
                "kernel": "fine Schur SpMV of the PCG step, q = A p with p.q (SELL-32x4, FP64, sell_spmv<double,3>)",
                "algorithmic_bytes_per_launch": int(alg),
                "algorithmic_bytes_rule": "nnz*(8+4) + 4(n+1) + 2*8*n (CSR index 4 B, value 8 B, x and y once)",
                "format_bytes_per_launch": int(fmt),
                "format_frac": round(fmt / (avg_launch_ms * 1e-3) / 1e9 / peak, 4),
                "avg_launch_ms": round(avg_launch_ms, 5), "launches": calls,
                "timed_in": f"profiled pass of {args.profile_steps} steps after the timed region"}

    # e2e: the public C ABI from host arrays: mesh -> setup -> device upload,
    # then per step (nds_simple_step_io) H2D of the state (u, p) from pinned
    # host memory, one SIMPLE iteration, D2H of the new state into the same
    # pinned arrays (the velocity read-back runs beside the pressure solve).
    # Projected like value, with the copies counted in the per-step part.
    e2e = None
    if args.e2e:
        import torch
        torch.cuda.set_device(local)
        del S
        t0 = time.perf_counter()
        mesh2 = N.Mesh.from_tetmesh(tm)
        P2 = N.Problem(mesh2, precision=prec, device=local, **OPTIONS)
        S2 = N.Solver(P2)
        fixed_s = time.perf_counter() - t0
        c = P2.counts()
        hu = [torch.zeros(c["nv"], dtype=torch.float64).pin_memory() for _ in range(3)]
        hp = torch.zeros(c["nc"], dtype=torch.float64).pin_memory()
        ptrs = [x.data_ptr() for x in hu] + [hp.data_ptr()]
        import ctypes as C
        L = N.lib()

        def e2e_step():
            r = N.IterReport()
            N._check(L.nds_simple_step_io(S2._h, *[C.c_void_p(p) for p in ptrs], *[C.c_void_p(p) for p in ptrs],
                                          C.byref(r)))
            return r
        for _ in range(args.warmup):
            e2e_step()
        e_outer, e_pcg, e_its = [], [], []
        for _ in range(args.steps):
            w = time.perf_counter()
            r = e2e_step()
            step_ms = (time.perf_counter() - w) * 1e3
            solve = r.ms_pressure - r.ms_refresh
            e_outer.append(step_ms - solve)
            e_pcg.append(solve)
            e_its.append(r.p_its)
        ev, _, _ = project(e_outer, e_pcg, e_its, prec)
        ev = _barrier_max(fixed_s + ev, ws, local)
        bytes_state = 8 * (3 * c["nv"] + c["nc"])
        e2e = {"value": round(ev, 3), "unit": "s", "h2d_bytes_per_step": bytes_state,
               "d2h_bytes_per_step": bytes_state, "fixed_setup_s": round(fixed_s, 3),
               "outer_ms": round(float(np.mean(e_outer)), 4)}
        P = P2

    cpu = None
    if rank == 0 and ws == 1 and args.cpu_baseline:
        cpu = cpu_baseline(P)
    if rank == 0:
        ss = STEADY_STATE[prec]
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(mean_ms, 4), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "f64/f32",
            "data": "synthetic (seeded pipe mesh)",
            "config": {"workload": f"{WORKLOAD}: straight pipe R=0.5 L=10, 1,231,200 tets (24x72 O-grid + 18x18 core, "
                                   f"100 slabs), Re=100, alpha_u=0.7, alpha_p=0.3, SA+cheb2 PCG rtol 1e-6",
                       "precision": f"{prec}: {PRECISION_NOTE[prec]}",
                       "cells": int(P.counts()["nc"]), "velocity_dofs": int(P.counts()["nv"]),
                       "step": "one SIMPLE outer iteration of the steady-state solve",
                       "projection": "N_outer x t_outer + N_pcg x t_pcg",
                       "steady_state_outer_iterations": ss["outer"], "steady_state_pcg_iterations": ss["pcg"],
                       "t_outer_ms": round(t_outer, 4), "t_pcg_ms": round(t_pcg, 5),
                       "timed_pcg_iterations_per_step": round(float(np.mean(pcg_its)), 2),
                       "steady_state_source": STEADY_STATE_SOURCE,
                       "l2": "working set per step > 126 MB L2 (fine operator ~1 GB); no flush",
                       "parallelism": "replicas" if ws > 1 else "single GPU", "host_setup_s": round(setup_s, 3),
                       "wall_ms_per_step": round(wall / args.steps * 1e3, 4)},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "kernel_ms_profiled_pass": {k: round(v[1], 3) for k, v in prof.items()},
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def _oracle_sample(P, threads, warmup, max_steps, max_seconds):
    """Time oracle steps; returns projected seconds, step times and the sample text."""
    from oracle.oracle import Oracle
    O = Oracle(P, threads=threads)
    for _ in range(warmup):
        O.step()
    t0 = time.perf_counter()
    outer, pcg, its, tot = [], [], [], []
    while len(tot) < max_steps and (time.perf_counter() - t0) < max_seconds:
        r = O.step()
        tot.append(r.ms_total)
        outer.append(r.ms_total - r.ms_pressure)
        pcg.append(r.ms_pressure)
        its.append(r.p_its)
    value, t_outer, t_pcg = project(outer, pcg, its, "fp64")
    sample = (f"{len(tot)} SIMPLE iterations of the {WORKLOAD} solve after {warmup} warm-up "
              f"({np.mean(tot) / 1e3:.3f} s each, {np.mean(its):.1f} PCG iterations each), projected as "
              f"N_outer x t_outer + N_pcg x t_pcg with t_outer {t_outer:.1f} ms, t_pcg {t_pcg:.1f} ms")
    return value, tot, sample


def cpu_baseline(P, max_seconds=25.0, max_steps=3):
    """The oracle (CPU FP64 restatement of the reference loop) on the host cores."""
    threads = os.cpu_count() or 1
    value, _, sample = _oracle_sample(P, threads, 1, max_steps, max_seconds)
    return {"value": round(value, 3), "unit": "s", "cores": threads, "kind": "port", "sample": sample}


def run_reference(args):
    """CPU reference arm: oracle/h8_oracle.c on the same workload (rank 0 only)."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    from nodals_b200 import meshgen
    from nodals_b200 import native as N
    P = N.Problem(N.Mesh.from_tetmesh(meshgen.named(WORKLOAD)), precision="fp64", **OPTIONS)
    threads = os.cpu_count() or 1
    warm = min(args.warmup, 1)
    value, tot, sample = _oracle_sample(P, threads, warm, args.steps, args.ref_seconds)
    value = round(value, 3) if WORKLOAD == "pipe1m" else 0.0
    ss = STEADY_STATE["fp64"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": ws,
            "steps": len(tot), "warmup": warm, "ms_per_step": round(float(np.mean(tot)), 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded pipe mesh)",
            "config": {"workload": f"{WORKLOAD} (as the CUDA arm)", "steady_state_outer_iterations": ss["outer"],
                       "steady_state_pcg_iterations": ss["pcg"],
                       "step": "one SIMPLE outer iteration (bounded sample)"},
            "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="nodals", choices=["nodals", "reference"])
    ap.add_argument("--precision", default="amg_fp32", choices=["amg_fp32", "fp64"])
    ap.add_argument("--workload", default=WORKLOAD, choices=["pipe1m", "pipe400k", "pipe40k"],
                    help="pipe1m is the benchmark; the smaller pipes serve kernel profiling only")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--ref-seconds", type=float, default=60.0)
    ap.add_argument("--profile-steps", type=int, default=3, help="profiled steps after the timed region")
    args = ap.parse_args()
    globals()["WORKLOAD"] = args.workload
    if args.warmup < 3 and args.impl == "nodals":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_nodals(args)


if __name__ == "__main__":
    main()
