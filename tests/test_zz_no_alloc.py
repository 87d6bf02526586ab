"""nds_continuity_noalloc: the continuity residual from caller-owned device
vectors with no allocation inside the library.

Checked against nds_simple_step on the same velocity: the norm must equal the
step's reported cont_norm bit for bit (same kernel, same fixed-order
reduction); r against a numpy evaluation of -(B u + fixedDiv) to 1e-12
relative.  Each input is evaluated by two calls in a row, so a scratch value
left over from the first call would show up in the second.  The device's free
memory (cudaMemGetInfo) and torch's allocator counters must not move across
the calls.  pipe400k has more cells than 1184 blocks x 256 threads, so the
grid-stride loop and every slot of the scratch array are used.  Collected
last (file name) and also run on its own.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

CFG = dict(max_outer=10, re=20.0, alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, amg_terminal=100)


def _fn(native):
    f = native.lib().nds_continuity_noalloc
    f.argtypes = [C.c_void_p] * 7
    f.restype = C.c_int
    return f


def _numpy_residual(P, u):
    ref = P.array("cell.ref").reshape(-1, 8)
    B = P.array("cell.bcoeff").reshape(-1, 8, 3)
    s = P.array("fixedDiv").copy()
    for a in range(8):
        g = ref[:, a]
        m = g >= 0
        for d in range(3):
            s[m] += B[m, a, d] * u[d][g[m]]
    return -s


@pytest.mark.gpu
@pytest.mark.parametrize("precision,mesh", [("fp64", "pipe_small"), ("amg_fp32", "pipe_small"),
                                            ("fp64", "pipe400k")])
def test_noalloc_continuity_matches_step(native, meshes, precision, mesh):
    import torch
    kw = dict(CFG, amg_terminal=300) if mesh == "pipe400k" else CFG
    P = native.Problem(native.Mesh.from_tetmesh(meshes(mesh)), precision=precision, **kw)
    if mesh == "pipe400k":
        assert P.counts()["nc"] > 1184 * 256
    S = native.Solver(P)
    f = _fn(native)
    for _ in range(2):
        rep = S.step()
        u0, u1, u2, p = S.fields()
        du = [torch.from_numpy(x).cuda() for x in (u0, u1, u2)]
        want_r = _numpy_residual(P, (u0, u1, u2))
        r = torch.full((len(p),), float("nan"), dtype=torch.float64, device="cuda")
        nrm = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        stats0 = torch.cuda.memory_stats()
        for _call in range(2):
            r.fill_(float("nan"))
            nrm.fill_(float("nan"))
            l0 = native.launch_count()
            st = f(S._h, *[C.c_void_p(x.data_ptr()) for x in du], C.c_void_p(r.data_ptr()),
                   C.c_void_p(nrm.data_ptr()), None)
            torch.cuda.synchronize()
            assert st == 0
            assert native.launch_count() - l0 == 3
            assert nrm.item() == rep.cont_norm
            got = r.cpu().numpy()
            assert np.linalg.norm(got - want_r) <= 1e-12 * np.linalg.norm(want_r)
        # nothing was allocated on the device by the two calls (the checks in
        # between only fill existing tensors and copy to the host)
        assert torch.cuda.mem_get_info()[0] == free0
        stats1 = torch.cuda.memory_stats()
        for key in ("allocation.all.allocated", "segment.all.allocated"):
            assert stats1.get(key, 0) == stats0.get(key, 0), key


@pytest.mark.gpu
def test_noalloc_continuity_rejects_fp32_state(native, meshes):
    import torch
    P = native.Problem(native.Mesh.from_tetmesh(meshes("pipe_tiny")), precision="fp32", **dict(CFG, amg_terminal=60))
    S = native.Solver(P)
    nv, nc = S.nv, S.nc
    u = [torch.zeros(nv, dtype=torch.float64, device="cuda") for _ in range(3)]
    r = torch.zeros(nc, dtype=torch.float64, device="cuda")
    nrm = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = _fn(native)(S._h, *[C.c_void_p(x.data_ptr()) for x in u], C.c_void_p(r.data_ptr()),
                     C.c_void_p(nrm.data_ptr()), None)
    assert st == -1
