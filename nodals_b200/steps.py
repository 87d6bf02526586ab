"""Run a few SIMPLE iterations of a benchmark configuration through the C ABI
and print the last iteration's report: the driver used for profiler captures
of single kernels (it does no complete solve and no timing of its own).

    python -m nodals_b200.steps --mesh pipe400k --steps 4 --config fast

Configurations: ``fast`` is the benchmark's fast path (precision mixed, PCG
inner solves, Galerkin guess over 4 corrections, FP16 fine operator in the
V-cycle); ``fp64`` and ``amg_fp32`` are the plain FP64 path and the FP32
V-cycle inside FP64 PCG.  The physical and solver controls are those of the
benchmark (Re 100, alpha_u 0.7, alpha_p 0.3, SA + Chebyshev(2), pressure
rtol 1e-6).  ``NDS_NO_GRAPHS=1`` in the environment makes the pressure loops
launch kernel by kernel, which profilers need to see them one by one.
"""
from __future__ import annotations

import argparse

from . import meshgen
from . import native as N

CONTROLS = dict(re=100.0, alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, run_mode="converge", simple_tol=1e-6,
                max_outer=100000, amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg")
CONFIGS = {
    "fast": dict(precision="mixed", p_krylov="pcg", p_guess=4, amg_half=1),
    "fp64": dict(precision="fp64"),
    "amg_fp32": dict(precision="amg_fp32"),
}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--mesh", default="pipe400k", help="a meshgen.named() mesh")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--config", default="fast", choices=sorted(CONFIGS))
    ns = ap.parse_args(argv)
    P = N.Problem(N.Mesh.from_tetmesh(meshgen.named(ns.mesh)), **dict(CONTROLS, **CONFIGS[ns.config]))
    S = N.Solver(P)
    r = None
    for _ in range(ns.steps):
        r = S.step()
    print(f"mesh {ns.mesh} config {ns.config}: iteration {r.it}, pressure iterations {r.p_its}, "
          f"relCont {r.rel_cont:.6e}", flush=True)


if __name__ == "__main__":
    main()
