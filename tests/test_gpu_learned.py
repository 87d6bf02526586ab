"""The learned stage inside the solver's FGMRES (precision mixed, learned=1).

* Fallback: a stage that never reduces the residual (a huge skip gain) is
  rejected at every application, and the run then equals the plain FGMRES
  run bit for bit (z = V(v) + 0).
* The trained parameters (nodals_b200/stage/mpnn_params.bin) on a held-out
  member of the seeded pipe family: every pressure solve meets the same FP64
  target p_rtol as the plain solve, so after 20 SIMPLE iterations the fields
  follow the plain run to 1e-5 (each solve differs within its tolerance), the
  stage is kept at most applications, and it takes fewer pressure
  iterations than the plain V-cycle.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

BASE = dict(alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, run_mode="converge", simple_tol=1e-12,
            max_outer=1000, amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg",
            precision="mixed", p_krylov="fgmres", p_restart=30)


def _pair(native, tm, re, params, iters, extra=None):
    mesh = native.Mesh.from_tetmesh(tm)
    out = []
    for learned in (0, 1):
        P = native.Problem(mesh, re=re, learned=learned, **dict(BASE, **(extra or {})))
        S = native.Solver(P)
        if learned:
            native.solver_load_stage(S, params)
        reps = [S.step() for _ in range(iters)]
        out.append((reps, S.fields(), native.solver_stage_counts(S) if learned else None))
    return out


def test_rejected_stage_equals_plain_fgmres(native, meshes):
    p = np.zeros(native.MPNN_NPARAM, dtype=np.float32)
    p[-1] = 1e6  # cs: out = 1e6 s, far from any correction
    (plain, fp, _), (stage, fs, counts) = _pair(native, meshes("pipe_small"), 20.0, p, 8,
                                                dict(amg_terminal=100))
    applied, fallbacks = counts
    assert applied > 0 and fallbacks == applied
    for a, b in zip(plain, stage):
        assert a.p_its == b.p_its and a.rel_cont == b.rel_cont and a.p_rel == b.p_rel
    for x, y in zip(fp, fs):
        assert np.array_equal(x, y)


def test_trained_stage_on_held_out_pipe(native):
    from nodals_b200 import meshgen
    from nodals_b200.stage import PARAMS, load_params
    if not PARAMS.exists():
        pytest.skip("no trained parameters")
    tm, re, _ = meshgen.family_member(meshgen.FAMILY_TRAIN)  # the first held-out member
    (plain, fp, _), (stage, fs, counts) = _pair(native, tm, re, load_params(), 20,
                                                dict(geom_from_inlet=1, amg_terminal=300))
    applied, fallbacks = counts
    assert applied > 0 and fallbacks < applied
    assert fallbacks <= applied // 10
    for a, b in zip(plain, stage):
        assert a.p_rel <= 1e-6 and b.p_rel <= 1e-6
        assert abs(a.rel_cont - b.rel_cont) <= 1e-4 * abs(a.rel_cont)
    for x, y in zip(fp, fs):
        assert rel_l2(y, x) <= 1e-5
    assert sum(b.p_its for b in stage) < sum(a.p_its for a in plain)
