"""Failure reporting of the device path, without faulting the GPU.

The pressure Krylov loop on the device is bounded by p_max; a solve that
misses its tolerance within that bound must come back as NDS_E_NOT_CONVERGED
(the reference throws "pressure solve failed requested inexact target",
h8_main_base.cu:2101), for both the device loop and the launch-by-launch
loop, and the same solver must stay usable afterwards (reset and run)."""
from __future__ import annotations

import pytest

CFG = dict(max_outer=10, re=20.0, alpha_u=0.7, alpha_p=0.3, amg_terminal=100)


@pytest.mark.gpu
@pytest.mark.parametrize("profiled", [False, True])
def test_pressure_cap_reports_not_converged(native, meshes, profiled):
    m = native.Mesh.from_tetmesh(meshes("pipe_small"))
    S = native.Solver(native.Problem(m, p_rtol=1e-12, p_max=2, **CFG))
    if profiled:
        S.profile(True)
    with pytest.raises(native.NdsError) as e:
        S.step()
    assert e.value.code == -5 and "pressure solve" in str(e.value)
    # the context and the handle stay usable
    ok = native.Solver(native.Problem(m, p_rtol=1e-6, p_max=400, **CFG))
    r = ok.step()
    assert r.p_its > 2 and r.rel_cont == 1.0
    S.reset()
    with pytest.raises(native.NdsError):
        S.step()
