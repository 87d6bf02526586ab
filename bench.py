#!/usr/bin/env python3
"""Benchmark of the steady SIMPLE hot path on one B200 (one process per GPU).

Workload (the benchmark metric's): the ~1M-tet straight pipe, O-grid 24 rings
x 72 sectors (+ an 18x18 square core) x 100 slabs, 6 tets per quad and slab =
1,231,200 tets, seed-1 jitter of +-5 % local spacing, Re = 100, alpha_u 0.7,
alpha_p 0.3, pressure rtol 1e-6 with the smoothed-aggregation AMG +
Chebyshev(2) V-cycle, converged when relCont <= 1e-6 and the pre-sweep
momentum audit <= 1e-6 (4193 SIMPLE iterations).

Metric: seconds to steady state.  ``value`` is a measured complete solve of
the fast configuration (FAST below: FP64 state, momentum and outer residual;
FP64 defect correction around FP32 inner Krylov solves with the FP32 V-cycle;
Galerkin initial guess over earlier pressure corrections), device-timed (the
sum of the per-iteration CUDA-event times of the SIMPLE loop) with the
problem already on the device.  The same solve runs through the public C ABI
from host arrays: ``e2e`` is its wall time from the host mesh arrays
(nds_mesh_from_arrays) through host setup, upload, the solve and the
read-back of the fields (nds_get_fields).  Then the plain FP64 path solves
the same problem (untimed) and the line states the relative L2 error of u,
v, w and p of the fast solve against it.

Steps: W warm-up and K timed SIMPLE iterations of the fast configuration on
a separate solver give ``ms_per_step`` (barrier + synchronize around the K
steps, max over ranks); a profiled pass of further iterations (per-kernel
CUDA events, launch-by-launch loops) times the roofline kernel live.  The
per-iteration working set (fine operator ~1 GB) is larger than the 126 MB
L2, so no flush is inserted.

Modes:
  python bench.py [--gpus N --steps K --warmup W]     this package (CUDA path)
  python bench.py --impl reference [...]                the CPU restatement of
      the reference's FP64 SIMPLE loop (oracle/, all host threads), same
      metric and workload, each step one SIMPLE iteration (bounded sample),
      projected to steady state with the FP64 iteration counts.
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
               max_outer=6000, amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg")
# the fast configuration of the metric
FAST = dict(precision="mixed", p_krylov="pcg", p_guess=4, amg_half=1)
FAST_NOTE = ("mixed: FP64 state, momentum, continuity and outer pressure residual; FP64 defect correction around "
             "FP32 inner PCG (FP32 operator copy for A p, FP64 reductions), inner rtol 1e-3; SA+cheb2 V-cycle in FP32 "
             "with its fine-level operator in FP16 (power-of-two scaled); Galerkin initial guess over the last 4 "
             "pressure corrections (stored products)")
# Complete FP64 solves of OPTIONS on WORKLOAD (tests/golden/cfg_pipe1m_re100_steady.npz,
# the reference's own run): outer and total PCG iterations, for the CPU projection.
STEADY_STATE_FP64 = {"outer": 4193, "pcg": 75316}


def project_fp64(outer_ms, pcg_ms, pcg_its):
    """Seconds to steady state of the FP64 loop from per-step times outside
    the pressure iterations (outer_ms), per-step pressure times (pcg_ms) and
    per-step pressure iteration counts (the CPU baseline's sample)."""
    ss = STEADY_STATE_FP64
    t_outer = float(np.mean(outer_ms))
    t_pcg = float(np.sum(pcg_ms)) / max(int(np.sum(pcg_its)), 1)
    return (ss["outer"] * t_outer + ss["pcg"] * t_pcg) / 1e3, t_outer, t_pcg


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic(key):
    """DRAM bytes of one launch from the committed ncu summary (scaled to the
    benchmark workload there), or None."""
    p = ROOT / "profiles" / "fine_spmv_traffic.json"
    if p.exists():
        return json.loads(p.read_text()).get(key)
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


def fine_spmv_bytes(problem, s: int, sx: int | None = None) -> float:
    """Compulsory bytes of one fine Schur SpMV in CSR terms: values (s B) and
    column indices (4 B) of every entry, row offsets, x and y once (sx B
    each; default s)."""
    sx = s if sx is None else sx
    row = problem.array("fine.row")
    n = len(row) - 1
    nnz = int(row[-1])
    return nnz * (s + 4) + 4 * (n + 1) + 2 * sx * n


def outer_kernel_bytes(problem) -> dict:
    """Compulsory bytes per SIMPLE iteration of the kernels outside the
    pressure solve, FP64 values (s = 8) and 4-byte indices, counted once per
    array with the actual counts: momentum assembly (reset, convection,
    finalize, B^T p, right-hand sides), one Gauss-Seidel sweep, the
    continuity residual, and the fine-operator refresh (FP64 values plus the
    FP32 and FP16 copies of the mixed path)."""
    s = 8
    c = problem.counts()
    nc, nv = c["nc"], c["nv"]
    zm = int(problem.array("mom.row")[-1])
    zp = int(problem.array("fine.row")[-1])
    zd = int(problem.array("fine.contribOff")[-1])
    return {
        "mom_assemble": 5 * s * zm + (172 + 48 * s) * nc + (12 + 25 * s) * nv,
        "mom_gs": (4 + s) * zm + (16 + 8 * s) * nv,
        "continuity": (48 * s + 36) * nc,
        "fine_refresh": (s + 4 + 2) * zp + 5 * zd + (24 * s + 8) * nc + s * nv,
    }


def outer_kernels(prof, kbytes, steps) -> dict | None:
    """Achieved algorithmic GB/s of the kernels outside the pressure solve in
    the profiled pass (CUDA events around their launches; the sweep runs
    beside the refresh on another stream, so both times include the
    contention), and their fraction of the measured copy bandwidth."""
    if steps <= 0:
        return None
    peak, kind = _peaks()
    out = {}
    for name, b in kbytes.items():
        calls, tot = prof.get(name, (0, 0.0))
        if calls == 0:
            continue
        ms = tot / steps
        gbs = b / (ms * 1e-3) / 1e9
        out[name] = {"ms_per_step": round(ms, 4), "algorithmic_bytes": int(b), "achieved_gbs": round(gbs, 1),
                     "frac": round(gbs / peak, 3)}
    out["peak_gbs"] = peak
    out["peak_kind"] = kind
    out["note"] = ("mom_gs and fine_refresh run concurrently on two streams; mom_assemble covers the cell and row "
                   "passes; bytes per the survey's per-kernel formulas with FP64 values")
    return out


def sell_format_bytes(problem, s: int, sx: int | None = None) -> float:
    """Bytes the SELL-32x4 fine operator actually streams per SpMV: padded
    values (s B) and 16-bit column deltas (slice width rounded up to a
    multiple of 4), slice offsets/widths, x and y (sx B each)."""
    sx = s if sx is None else sx
    row = problem.array("fine.row")
    n = len(row) - 1
    lens = np.diff(row)
    ns = (n + 31) // 32
    w = np.zeros(ns * 32, dtype=np.int64)
    w[:n] = lens
    widths = (w.reshape(ns, 32).max(axis=1) + 3) // 4 * 4
    padded = int(widths.sum()) * 32
    return padded * (s + 2) + 8 * ns + 2 * sx * n


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_nodals(args):
    from nodals_b200 import meshgen
    from nodals_b200 import native as N
    ws, rank, local = _dist()
    if ws > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=900))
    tm = meshgen.named(WORKLOAD)
    fast = dict(OPTIONS, **FAST, device=local)
    stage = None
    if fast.get("learned"):
        from nodals_b200.stage import load_params
        stage = load_params()

    # --- per-iteration timing (warm-up, K timed steps, profiled steps) -------
    P = N.Problem(N.Mesh.from_tetmesh(tm), **fast)
    S = N.Solver(P)
    if stage is not None:
        N.solver_load_stage(S, stage)
    for _ in range(args.warmup):
        S.step()
    l0 = N.launch_count()
    _barrier_max(0.0, ws, local)
    with Clocks(local) as clk:
        dev_ms, p_its = [], []
        for _ in range(args.steps):
            r = S.step()
            dev_ms.append(r.ms_assembly + r.ms_momentum + r.ms_continuity + r.ms_pressure + r.ms_update)
            p_its.append(r.p_its)
        step_launches = N.launch_count() - l0
        mean_ms = _barrier_max(float(np.mean(dev_ms)), ws, local)
        # profiled pass: per-kernel CUDA events need the launch-by-launch loops
        S.profile(True)
        for _ in range(args.profile_steps):
            S.step()
        prof = S.profile_read()
        S.profile(False)
        counts = P.counts()
        kbytes = outer_kernel_bytes(P)
        del S, P

        # --- the metric: a complete solve through the C ABI from host arrays --
        _barrier_max(0.0, ws, local)
        l1 = N.launch_count()
        w0 = time.perf_counter()
        mesh = N.Mesh.from_tetmesh(tm)
        P = N.Problem(mesh, **fast)
        S = N.Solver(P)
        if stage is not None:
            N.solver_load_stage(S, stage)
        setup_s = time.perf_counter() - w0
        rep = S.solve()
        fields = S.fields()
        e2e_s = time.perf_counter() - w0
        solve_launches = N.launch_count() - l1
    value = _barrier_max(rep.loop_ms / 1e3, ws, local)
    e2e_s = _barrier_max(e2e_s, ws, local)
    if not rep.converged:
        raise RuntimeError(f"the fast solve did not converge ({rep.outer_its} iterations)")
    del S

    # --- roofline: the dominant kernel, the V-cycle's fine-level SELL SpMV --
    # (FP16 values, FP32 vectors: 4 per inner iteration); the inner Krylov
    # product (FP32 values) and the FP64 defect product are reported beside it
    roof = None
    half = bool(FAST.get("amg_half"))
    cat = "fine_spmv_half" if half else "fine_spmv_amg"
    calls, tot = prof[cat]
    peak, peak_kind = _peaks()

    def side(name, s_val, s_vec):
        c, t = prof[name]
        if c == 0:
            return None
        return {"avg_launch_ms": round(t / c, 5), "launches": c,
                "achieved": round(fine_spmv_bytes(P, s_val, s_vec) / (t / c * 1e-3) / 1e9, 1)}
    if args.profile_steps > 0 and calls > 0:
        avg_ms = tot / calls
        sv = 2 if half else 4
        alg = fine_spmv_bytes(P, sv, 4)
        fmt = sell_format_bytes(P, sv, 4)
        achieved = alg / (avg_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": _traffic("bytes_per_launch_pipe1m_half" if half else "bytes_per_launch_pipe1m_fp32"),
                "peak_kind": peak_kind,
                "kernel": ("fine Schur SELL-32x4 SpMV of the V-cycle (sell_spmv<float,*,*,__half>: FP16 values, "
                           "16-bit column deltas, FP32 vectors): fine-level smoothing and residual steps") if half else
                          "fine Schur SELL-32x4 SpMV in FP32 (sell_spmv<float,*>)",
                "algorithmic_bytes_per_launch": int(alg),
                "algorithmic_bytes_rule": f"nnz*({sv}+4) + 4(n+1) + 2*4*n (CSR index 4 B, value {sv} B, x and y once)",
                "format_bytes_per_launch": int(fmt),
                "format_frac": round(fmt / (avg_ms * 1e-3) / 1e9 / peak, 4),
                "avg_launch_ms": round(avg_ms, 5), "launches": calls,
                "timed_in": f"profiled pass of {args.profile_steps} steps after the timed steps",
                "inner_krylov_spmv_fp32": side("fine_spmv_amg", 4, 4),
                "fp64_defect_spmv": side("fine_spmv", 8, 8)}

    # --- field error against the plain FP64 path (untimed) -------------------
    errors = None
    if args.fp64_check:
        P64 = N.Problem(mesh, **dict(OPTIONS, precision="fp64", device=local))
        S64 = N.Solver(P64)
        r64 = S64.solve()
        f64 = S64.fields()
        errors = {"u": _rel(fields[0], f64[0]), "v": _rel(fields[1], f64[1]), "w": _rel(fields[2], f64[2]),
                  "p": _rel(fields[3], f64[3]), "fp64_outer_its": r64.outer_its,
                  "fp64_loop_s": round(r64.loop_ms / 1e3, 3),
                  "speedup_vs_fp64_loop": round(r64.loop_ms / rep.loop_ms, 3)}
        del S64, P64

    cpu = None
    if rank == 0 and ws == 1 and args.cpu_baseline:
        cpu = cpu_baseline(N.Problem(N.Mesh.from_tetmesh(tm), **dict(OPTIONS, precision="fp64")))
    if rank == 0:
        nbytes_in = tm.points.nbytes + tm.tets.astype(np.int32).nbytes + tm.bfaces.astype(np.int32).nbytes \
            + tm.btag.astype(np.int32).nbytes
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(mean_ms, 4), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64/f32", "data": "synthetic (seeded pipe mesh)",
            "config": {"workload": f"{WORKLOAD}: straight pipe R=0.5 L=10, 1,231,200 tets (24x72 O-grid + 18x18 "
                                   f"core, 100 slabs), Re=100, alpha_u=0.7, alpha_p=0.3, SA+cheb2 V-cycle, "
                                   f"pressure rtol 1e-6, steady state at relCont and momentum audit <= 1e-6",
                       "precision": FAST_NOTE, "krylov": FAST.get("p_krylov", "pcg"),
                       "learned_stage": bool(FAST.get("learned")),
                       "cells": int(counts["nc"]), "velocity_dofs": int(counts["nv"]),
                       "value_is": "device time of one complete solve (sum of the per-iteration CUDA-event times)",
                       "steady_state_outer_iterations": int(rep.outer_its),
                       "avg_pressure_iterations": round(rep.avg_pressure_its, 3),
                       "pressure_s": round(rep.pressure_ms / 1e3, 3),
                       "step": "one SIMPLE outer iteration (ms_per_step: K timed iterations after W warm-up)",
                       "timed_steps_pressure_iterations": round(float(np.mean(p_its)), 2),
                       "l2": "working set per step > 126 MB L2 (fine operator ~1 GB); no flush",
                       "parallelism": "replicas" if ws > 1 else "single GPU", "host_setup_s": round(setup_s, 3)},
            "field_rel_l2_vs_fp64": errors,
            "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_s, 3), "unit": "s", "h2d_bytes_per_step": int(nbytes_in),
                    "d2h_bytes_per_step": int(8 * (3 * counts["nv"] + counts["nc"])),
                    "what": "wall time of mesh host arrays -> host setup -> device upload -> complete solve -> "
                            "fields read back to host, through the C ABI (ctypes); h2d counts the mesh arrays "
                            "passed in (the library uploads its setup from them), d2h the fields"},
            "gpu_launches": int(step_launches),
            "gpu_launches_complete_solve": int(solve_launches),
            "clocks": clk.summary(),
            "kernel_ms_profiled_pass": {k: round(v[1], 3) for k, v in prof.items()},
            "outer_kernels": outer_kernels(prof, kbytes, args.profile_steps),
            "simple_its_per_s": round(rep.outer_its / max(rep.loop_ms / 1e3, 1e-9), 2),
            "pressure_ms_per_outer_iteration": round(rep.pressure_ms / max(rep.outer_its, 1), 3),
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
    value, t_outer, t_pcg = project_fp64(outer, pcg, its)
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
    ss = STEADY_STATE_FP64
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
    ap.add_argument("--workload", default=WORKLOAD, choices=["pipe1m", "pipe400k", "pipe40k"],
                    help="pipe1m is the benchmark; the smaller pipes serve kernel profiling only")
    ap.add_argument("--no-fp64-check", dest="fp64_check", action="store_false",
                    help="skip the FP64 solve that gives the field errors")
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
