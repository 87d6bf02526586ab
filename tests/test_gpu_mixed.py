"""Mixed-precision pressure path (precision "mixed": FP32 inner PCG or FGMRES
inside an FP64 defect-correction loop, optional Galerkin initial guess) on
the GPU, against the FP64 path.

Every pressure solve of the mixed path meets the same FP64 target as the FP64
path (||b - A x|| <= p_rtol ||b|| on the FP64 operator), so the SIMPLE
iterates follow the FP64 ones to about p_rtol.  Tolerances: relCont 1e-5
relative per iteration, fields 1e-6 relative L2 after 10 iterations, every
reported pressure residual <= p_rtol.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

CFG = dict(re=20.0, alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, amg_terminal=100, max_outer=10,
           amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg")
VARIANTS = {
    "pcg": dict(p_krylov="pcg"),
    "pcg_tight": dict(p_krylov="pcg", p_inner_rtol=1e-6),
    "fgmres": dict(p_krylov="fgmres", p_restart=30),
    "fgmres_short": dict(p_krylov="fgmres", p_restart=5),
    "pcg_guess2": dict(p_krylov="pcg", p_guess=2),
    "fgmres_guess1": dict(p_krylov="fgmres", p_guess=1),
    "pcg_guess4_fresh": dict(p_krylov="pcg", p_guess=4, p_guess_fresh=1),
    "pcg_half_guess4": dict(p_krylov="pcg", p_guess=4, amg_half=1),
    "fgmres_half": dict(p_krylov="fgmres", amg_half=1),
}


def _solver(native, meshes, mesh="pipe_small", **kw):
    P = native.Problem(native.Mesh.from_tetmesh(meshes(mesh)), **dict(CFG, **kw))
    return P, native.Solver(P)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_mixed_tracks_fp64(native, meshes, variant):
    _, S64 = _solver(native, meshes)
    _, Sm = _solver(native, meshes, precision="mixed", **VARIANTS[variant])
    for _ in range(10):
        a, b = S64.step(), Sm.step()
        assert b.p_rel <= 1e-6, (b.it, b.p_rel)
        assert abs(a.rel_cont - b.rel_cont) <= 1e-5 * abs(a.rel_cont), (a.it, a.rel_cont, b.rel_cont)
    for x, y in zip(S64.fields(), Sm.fields()):
        assert rel_l2(y, x) <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["pcg", "fgmres_guess1", "pcg_half_guess4"])
def test_mixed_is_deterministic_and_graph_equals_host_loop(native, meshes, variant):
    """Two solvers give bitwise-equal runs; the device loops (conditional
    graphs) and the launch-by-launch loops taken while the profiler is on
    launch the same kernels in the same order."""
    P, A = _solver(native, meshes, precision="mixed", **VARIANTS[variant])
    B = native.Solver(P)
    C = native.Solver(P)
    C.profile(True)
    for _ in range(6):
        a, b, c = A.step(), B.step(), C.step()
        assert a.p_its == b.p_its == c.p_its and a.rel_cont == b.rel_cont == c.rel_cont
        assert a.p_rel == b.p_rel == c.p_rel
    for x, y, z in zip(A.fields(), B.fields(), C.fields()):
        assert np.array_equal(x, y) and np.array_equal(x, z)


@pytest.mark.gpu
def test_galerkin_guess_saves_iterations(native, meshes):
    """Later in a solve the pressure corrections of successive SIMPLE
    iterations are nearly parallel, so the Galerkin guess over the last two
    cuts the inner iterations (same FP64 target)."""
    kw = dict(max_outer=60, run_mode="converge", simple_tol=1e-12)
    _, S0 = _solver(native, meshes, precision="mixed", p_krylov="pcg", **kw)
    _, S2 = _solver(native, meshes, precision="mixed", p_krylov="pcg", p_guess=2, **kw)
    its0 = its2 = 0
    for k in range(60):
        a, b = S0.step(), S2.step()
        if k >= 20:
            its0 += a.p_its
            its2 += b.p_its
        assert a.p_rel <= 1e-6 and b.p_rel <= 1e-6
    assert its2 < its0, (its0, its2)
