"""Pin the CPU oracle (oracle/h8_oracle.c) against the reference H8 binaries.

tests/golden/run_*.npz hold the SIMPLE history (relCont printed with 12
digits, pressure iteration counts) and the final VTU fields (P0 pressure and
cell-average velocity, 17 digits) of the reference FP64 solver run on the
same seeded meshes (tests/golden/make_golden.py).  The oracle, fed with the
product's host setup (itself pinned by test_setup_parity.py), must reproduce
them: relCont to 1e-8 relative (the printed precision is 1e-12), identical
pressure iteration counts, fields to relative L2 1e-8.  SUPG runs (no VTU in
the reference's SUPG entry) are compared through the analytic-error line
(errors against Hagen-Poiseuille, pressure-drop fit) and at 1e-7: the
reference's default SUPG kernel evaluates its quadrature terms in FP32.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2
from test_gpu_parity import SUPG_TOL, _options_from_cmd, check_hp

MESH = {"tiny": "pipe_tiny", "small": "pipe_small", "m40k": "pipe40k"}


def _cases():
    out = []
    for p in sorted(GOLDEN.glob("run_*.npz")):
        case = p.stem[4:]
        if case.endswith("fp32") or case.startswith("m40k"):
            continue  # the oracle is FP64; the 48k case is covered on the GPU
        out.append(case)
    return out


@pytest.mark.parametrize("case", _cases())
def test_oracle_matches_reference_run(native, oracle_mod, meshes, case):
    g = np.load(GOLDEN / f"run_{case}.npz")
    opts = _options_from_cmd(str(g["cmd"]))
    P = native.Problem(native.Mesh.from_tetmesh(meshes(MESH[case.split("_")[0]])), **opts)
    O = oracle_mod.Oracle(P)
    tol = SUPG_TOL if opts.get("supg") else 1e-8
    idx = {int(i): k for k, i in enumerate(g["it"])}
    for it in range(1, int(g["it"].max()) + 1):
        r = O.step()
        if it in idx:
            k = idx[it]
            assert abs(r.rel_cont - g["rel_cont"][k]) <= tol * abs(g["rel_cont"][k]), (it, r.rel_cont, g["rel_cont"][k])
            assert r.p_its == int(g["p_its"][k]), (it, r.p_its, int(g["p_its"][k]))
    u0, u1, u2, p = O.fields()
    if "p" in g.files:
        uc = native.cell_average_velocity(P, u0, u1, u2)
        assert rel_l2(p, g["p"]) <= 1e-8
        assert rel_l2(uc, g["u_cell"]) <= 1e-8
    if "hp" in g.files:
        check_hp(native.hp_errors(P, u0, u1, u2, p), g["hp"], tol)
