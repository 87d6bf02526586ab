"""nds_simple_step_io: one SIMPLE iteration with the state passed through
host memory gives bitwise the result of nds_set_fields + nds_simple_step +
nds_get_fields -- with page-locked outputs (velocity read back beside the
pressure solve, inputs aliasing outputs) and with pageable ones -- and
reports a failed pressure solve with the same status."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN  # noqa: F401  (conftest on the path)

CFG = dict(re=20.0, alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, amg_terminal=100,
           amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg", max_outer=10)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "amg_fp32", "fp32"])
def test_step_io_matches_set_step_get(native, meshes, precision):
    import torch
    P = native.Problem(native.Mesh.from_tetmesh(meshes("pipe_small")), precision=precision, **CFG)
    c = P.counts()
    sizes = (c["nv"], c["nv"], c["nv"], c["nc"])
    A, B, D = native.Solver(P), native.Solver(P), native.Solver(P)
    pinned = [torch.zeros(n, dtype=torch.float64).pin_memory() for n in sizes]
    pageable = [np.zeros(n) for n in sizes]
    for _ in range(6):
        ra = A.step()
        rb = B.step_io([t.data_ptr() for t in pinned], [t.data_ptr() for t in pinned])
        rd = D.step_io(pageable, pageable)
        for r in (rb, rd):
            assert (r.p_its, r.rel_cont, r.p_rel, r.cont_norm) == (ra.p_its, ra.rel_cont, ra.p_rel, ra.cont_norm)
        fa = A.fields()
        for x, y, z in zip(fa, pinned, pageable):
            assert np.array_equal(x, y.numpy()) and np.array_equal(x, z)


@pytest.mark.gpu
def test_step_io_reports_pressure_failure(native, meshes):
    import torch
    P = native.Problem(native.Mesh.from_tetmesh(meshes("pipe_small")), **dict(CFG, p_max=1, p_rtol=1e-12))
    S = native.Solver(P)
    c = P.counts()
    out = [torch.zeros(n, dtype=torch.float64).pin_memory() for n in (c["nv"], c["nv"], c["nv"], c["nc"])]
    with pytest.raises(native.NdsError) as e:
        S.step_io([None] * 4, [t.data_ptr() for t in out])
    assert e.value.code == -5
