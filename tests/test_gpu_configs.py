"""Parity on the two benchmark configurations, against the reference H8 FP64
binary's own runs (fixtures tests/golden/cfg_*.npz, made on a B200 by
``tests/golden/make_golden.py --configs``; reference loop
gpu/serial_cuda/h8_main_base.cu:2046-2119, print cadence :2115-2117).

* ~40k-tet pipe (47,880 cells), Re 20, alpha_u 0.7, alpha_p 0.3, SA + cheb2
  PCG rtol 1e-6, 300 outer iterations: relCont at every printed iteration to
  1e-8 relative (+ 1e-16 absolute, the rounding level of relCont(1) = 1),
  equal PCG counts, P0 pressure and cell-average velocity to
  1e-8 relative L2, the analytic-error line to 1e-8.
* ~1M-tet pipe (1,231,200 cells), Re 100, converge at 1e-6 (relCont and the
  momentum audit): the same 4193 outer iterations, relCont at every printed
  iteration to 1e-8 relative, equal PCG counts, sampled fields (every 61st
  cell) and the full-field norms to 1e-8.  The amg_fp32 and mixed-precision
  solves of the same configuration reach fields within 1e-6 relative L2 of
  the FP64 solve, per component (u, v, w of the cell-average velocity and p).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

SA = dict(amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg")
CFG1 = dict(re=20.0, alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, run_mode="converge", simple_tol=1e-12,
            max_outer=300, **SA)
CFG2 = dict(re=100.0, alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, run_mode="converge", simple_tol=1e-6,
            max_outer=6000, **SA)
# the benchmark's fast path (bench.py)
MIXED = dict(precision="mixed", p_krylov="pcg", p_guess=4, amg_half=1)


def _history(S, n_max, printed):
    """Step up to n_max times (stopping at convergence); keep the reports of
    the printed iterations."""
    got = {}
    last = None
    for _ in range(n_max):
        r = S.step()
        if r.it in printed:
            got[r.it] = (r.rel_cont, r.p_its)
        last = r
        if r.converged:
            break
    return got, last


def _cell_fields(native, P, S):
    u0, u1, u2, p = S.fields()
    uc = np.zeros((P.counts()["nc"], 3))
    native.cell_average_velocity(P, u0, u1, u2, uc)
    return p, uc, (u0, u1, u2)


def _check_history(g, got, tol=1e-8, floor=1e-16):
    """relCont is the continuity residual over the first iteration's, so
    relCont(1) = 1 and floor is the FP64 rounding level of that residual:
    near steady state (relCont ~ 1e-9) the two solvers' different, each
    deterministic, reduction orders leave differences of ~5e-17 there."""
    for it, rel, pcg in zip(g["it"], g["rel_cont"], g["p_its"]):
        r, k = got[int(it)]
        assert abs(r - rel) <= tol * abs(rel) + floor, (int(it), r, float(rel))
        assert k == int(pcg), (int(it), k, int(pcg))


@pytest.mark.gpu
def test_config1_pipe40k_fp64_matches_reference(native, meshes):
    g = np.load(GOLDEN / "cfg_pipe40k_re20_300.npz")
    P = native.Problem(native.Mesh.from_tetmesh(meshes("pipe40k")), **CFG1)
    S = native.Solver(P)
    got, last = _history(S, 300, set(int(i) for i in g["it"]))
    assert last.it == 300
    _check_history(g, got)
    p, uc, u = _cell_fields(native, P, S)
    assert rel_l2(p, g["p"]) <= 1e-8
    assert rel_l2(uc, g["u_cell"]) <= 1e-8
    hp = native.hp_errors(P, *u, p)
    for key, want in zip(("h_eff", "u_l2", "u_rel_l2", "p_shifted_l2", "p_shifted_rel_l2", "pressure_shift",
                          "dp_fit"), g["hp"]):
        assert abs(hp[key] - want) <= 1e-8 * abs(want) + 1e-12, (key, hp[key], want)


@pytest.fixture(scope="module")
def pipe1m(native, meshes):
    mesh = native.Mesh.from_tetmesh(meshes("pipe1m"))
    g = np.load(GOLDEN / "cfg_pipe1m_re100_steady.npz")
    P = native.Problem(mesh, **CFG2)
    S = native.Solver(P)
    got, last = _history(S, 6000, set(int(i) for i in g["it"]))
    p, uc, _ = _cell_fields(native, P, S)
    del S
    return dict(mesh=mesh, g=g, got=got, last=last, p=p, uc=uc, P=P)


@pytest.mark.gpu
def test_config2_pipe1m_fp64_matches_reference(pipe1m):
    g, last = pipe1m["g"], pipe1m["last"]
    assert last.converged and last.it == int(g["fullconv"][0]) == 4193
    _check_history(g, pipe1m["got"])
    s = int(g["field_stride"][0])
    p, uc = pipe1m["p"], pipe1m["uc"]
    assert rel_l2(p[::s], g["p_sample"]) <= 1e-8
    assert rel_l2(uc[::s], g["u_cell_sample"]) <= 1e-8
    assert abs(np.linalg.norm(p) - g["p_norm"][0]) <= 1e-8 * g["p_norm"][0]
    for d in range(3):
        assert abs(np.linalg.norm(uc[:, d]) - g["u_cell_norm"][d]) <= 1e-8 * g["u_cell_norm"][d]


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["amg_fp32", "mixed"])
def test_config2_pipe1m_fast_paths_match_fp64_fields(native, pipe1m, variant):
    kw = dict(precision="amg_fp32") if variant == "amg_fp32" else MIXED
    P = native.Problem(pipe1m["mesh"], **dict(CFG2, **kw))
    S = native.Solver(P)
    rep = S.solve()
    assert rep.converged
    p, uc, _ = _cell_fields(native, P, S)
    for d in range(3):
        assert rel_l2(uc[:, d], pipe1m["uc"][:, d]) <= 1e-6, d
    assert rel_l2(p, pipe1m["p"]) <= 1e-6
