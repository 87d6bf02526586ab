"""What the learned stage gains: held-out members of the pipe family (and
optionally the benchmark pipe), each solved for a number of SIMPLE
iterations by the mixed-precision FGMRES pressure solve with and without the
learned stage (same FP64 pressure target p_rtol).  Per case: pressure
iterations, pressure-stage device time, stage applications and fallbacks,
the largest pressure residual, and the relative L2 difference of the final
fields.

    python -m nodals_b200.stage.evaluate [--members 64 65 ...] [--pipe1m] [--iters 60] [--params FILE]

With --pipe1m-solve (and --members with no value), the benchmark pipe is
solved to steady state instead (the benchmark's controls: Re 100, converge
at 1e-6; FGMRES(30), Galerkin guess over 4 corrections, FP16 V-cycle), with
and without the stage.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from .. import meshgen
from .. import native as N
from . import load_params

SOLVER = dict(alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, run_mode="converge", simple_tol=1e-12,
              max_outer=100000, amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg",
              precision="mixed", p_krylov="fgmres", p_restart=30, amg_terminal=300)


def compare(tm, re, params, iters, geom_from_inlet=1, **extra):
    mesh = N.Mesh.from_tetmesh(tm)
    out = {}
    fields = {}
    for learned in (0, 1):
        P = N.Problem(mesh, re=re, learned=learned, geom_from_inlet=geom_from_inlet, **dict(SOLVER, **extra))
        S = N.Solver(P)
        if learned:
            N.solver_load_stage(S, params)
        its, ms, prel = 0, 0.0, 0.0
        for _ in range(iters):
            r = S.step()
            its += r.p_its
            ms += r.ms_pressure
            prel = max(prel, r.p_rel)
        applied, fallback = N.solver_stage_counts(S)
        fields[learned] = S.fields()
        out["learned" if learned else "plain"] = dict(p_its=its, pressure_ms=round(ms, 3), max_p_rel=prel,
                                                     stage_applied=applied, stage_fallbacks=fallback)
    out["field_rel_l2"] = [float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
                           for a, b in zip(fields[1], fields[0])]
    out["its_ratio"] = out["learned"]["p_its"] / max(out["plain"]["p_its"], 1)
    out["time_ratio"] = out["learned"]["pressure_ms"] / max(out["plain"]["pressure_ms"], 1e-9)
    return out


# the benchmark's controls (bench.py) with FGMRES(30) inner solves
BENCH = dict(re=100.0, alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, run_mode="converge", simple_tol=1e-6,
             max_outer=6000, amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg",
             precision="mixed", p_krylov="fgmres", p_restart=30, p_guess=4, amg_half=1)


def solve_pipe1m(params):
    """Complete solves of the benchmark pipe without and with the stage."""
    mesh = N.Mesh.from_tetmesh(meshgen.named("pipe1m"))
    out, fields = {}, {}
    for learned in (0, 1):
        P = N.Problem(mesh, learned=learned, **BENCH)
        S = N.Solver(P)
        if learned:
            N.solver_load_stage(S, params)
        r = S.solve()
        applied, fallback = N.solver_stage_counts(S) if learned else (0, 0)
        fields[learned] = S.fields()
        out["learned" if learned else "plain"] = dict(
            outer=r.outer_its, converged=bool(r.converged), avg_p_its=r.avg_pressure_its,
            loop_s=round(r.loop_ms / 1e3, 3), pressure_s=round(r.pressure_ms / 1e3, 3), stage_applied=applied,
            stage_fallbacks=fallback)
        del S, P
    out["field_rel_l2"] = [float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
                           for a, b in zip(fields[1], fields[0])]
    out["time_ratio"] = out["learned"]["loop_s"] / max(out["plain"]["loop_s"], 1e-9)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--members", type=int, nargs="*",
                    default=list(range(meshgen.FAMILY_TRAIN, meshgen.FAMILY_TRAIN + meshgen.FAMILY_HELD_OUT)))
    ap.add_argument("--iters", type=int, default=60)
    ap.add_argument("--pipe1m", action="store_true")
    ap.add_argument("--pipe1m-solve", action="store_true", help="complete solves of the benchmark pipe")
    ap.add_argument("--params")
    ns = ap.parse_args()
    params = load_params(ns.params)
    if ns.pipe1m_solve:
        r = solve_pipe1m(params)
        r.update(case="pipe1m complete solve")
        print(json.dumps(r), flush=True)
    rows = []
    for i in ns.members:
        tm, re, prm = meshgen.family_member(i)
        r = compare(tm, re, params, ns.iters)
        r.update(case=f"member {i}", **prm)
        rows.append(r)
        print(json.dumps(r), flush=True)
    if ns.pipe1m:
        r = compare(meshgen.named("pipe1m"), 100.0, params, ns.iters, geom_from_inlet=0)
        r.update(case="pipe1m")
        rows.append(r)
        print(json.dumps(r), flush=True)
    fam = [r for r in rows if r["case"].startswith("member")]
    if fam:
        print(json.dumps({"summary": "held-out members", "n": len(fam),
                          "its_ratio_mean": float(np.mean([r["its_ratio"] for r in fam])),
                          "time_ratio_mean": float(np.mean([r["time_ratio"] for r in fam]))}), flush=True)


if __name__ == "__main__":
    main()
