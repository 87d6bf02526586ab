"""The learned stage's CUDA kernels (tcgen05 BF16 GEMMs with TMEM
accumulators, FP32 gathers, FP64 reductions) against the CPU oracle
oracle/mpnn.py, through the C ABI.

Tolerances: the oracle rounds to BF16 at the same points as the kernels but
sums in float64 where the tensor core sums in FP32, so a few BF16 roundings
differ by one unit (2^-8 relative); z and the loss agree to 2e-3 relative
(L2), every parameter-gradient block to 2e-2 relative (L2), stored
activations differ in at most 1 % of their values.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def face_graph(native, meshes, name):
    """The face graph of a pipe mesh's cells, with random symmetric negative
    edge weights (the scaled pressure operator's sign pattern) and a random
    positive scaling."""
    tm = meshes(name)
    m = native.Mesh.from_tetmesh(tm)
    P = native.Problem(m, max_outer=10, re=20.0, alpha_u=0.7, alpha_p=0.3, amg_terminal=100)
    tets = P.array("mesh.tets").reshape(-1, 4)
    n = len(tets)
    faces = {}
    for c in range(n):
        t = sorted(tets[c])
        for skip in range(4):
            key = tuple(v for q, v in enumerate(t) if q != skip)
            faces.setdefault(key, []).append(c)
    rng = np.random.default_rng(7)
    nbr = -np.ones((n, 4), dtype=np.int32)
    ew = np.zeros((n, 4), dtype=np.float32)
    cnt = np.zeros(n, dtype=int)
    for cells in faces.values():
        if len(cells) == 2:
            a, b = cells
            w = -0.05 - 0.25 * rng.random()
            nbr[a, cnt[a]], ew[a, cnt[a]] = b, w
            nbr[b, cnt[b]], ew[b, cnt[b]] = a, w
            cnt[a] += 1
            cnt[b] += 1
    dscale = (0.5 + rng.random(n)).astype(np.float32)
    return nbr, ew, dscale


def _dev(torch, a):
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    torch.cuda.synchronize()  # the library runs on its own streams
    return t


@pytest.mark.parametrize("mesh,segs", [("pipe_tiny", None), ("pipe_small", "two")])
def test_forward_matches_oracle(native, meshes, mesh, segs):
    import torch
    from oracle import mpnn as M
    nbr, ew, dscale = face_graph(native, meshes, mesh)
    n = len(nbr)
    seg = None if segs is None else [0, n // 3, n]
    rng = np.random.default_rng(1)
    v = rng.normal(size=n).astype(np.float32)
    p = M.init_params(2)
    net = native.Mpnn(n, training=True)
    net.set_params(p)
    # the graph holds raw device addresses: keep the tensors alive
    keep = [_dev(torch, nbr), _dev(torch, ew), _dev(torch, dscale)]
    g = net.graph(n, *keep)
    vd = _dev(torch, v)
    z = torch.zeros(n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    net.forward(g, vd, z, seg)
    torch.cuda.synchronize()
    zo, cache = M.forward(p, nbr, ew, dscale, v, seg)
    assert rel_l2(z.cpu().numpy(), zo) <= 2e-3
    # stored activations h1, h2, h3 (BF16): nearly all values bitwise equal
    buf = torch.zeros((n, 64), dtype=torch.bfloat16, device="cuda")
    for layer in (1, 2):
        net.activations(layer, buf)
        got = buf.float().cpu().numpy()
        want = cache["h"][layer]
        assert np.mean(got != want) <= 0.01, (layer, np.mean(got != want))
        assert rel_l2(got, want) <= 5e-3
    del keep


@pytest.mark.parametrize("mesh", ["pipe_tiny", "pipe_small"])
def test_gradients_match_oracle(native, meshes, mesh):
    import torch
    from oracle import mpnn as M
    nbr, ew, dscale = face_graph(native, meshes, mesh)
    n = len(nbr)
    seg = [0, n // 2, n]
    rng = np.random.default_rng(4)
    v = rng.normal(size=n).astype(np.float32)
    x = rng.normal(size=n).astype(np.float32)
    p = M.init_params(6)
    net = native.Mpnn(n, training=True)
    net.set_params(p)
    keep = [_dev(torch, nbr), _dev(torch, ew), _dev(torch, dscale)]
    g = net.graph(n, *keep)
    vd, xd = _dev(torch, v), _dev(torch, x)
    loss = net.loss_backward(g, vd, xd, seg)
    grads = net.grads()
    lo, go, _ = M.loss_grad(p, nbr, ew, dscale, v, x, seg)
    assert abs(loss - lo) <= 2e-3 * abs(lo)
    blocks = {"We": (M.OFF_WE, 128), "be": (M.OFF_BE, 64), "wd": (M.OFF_WD, 64), "bd/cs": (M.OFF_BD, 2)}
    for l in (1, 2, 3):
        blocks[f"W{l}"] = (M.off_w(l), 64 * 128)
        blocks[f"b{l}"] = (M.off_b(l), 64)
    for name, (o, k) in blocks.items():
        assert rel_l2(grads[o:o + k], go[o:o + k]) <= 2e-2, (name, rel_l2(grads[o:o + k], go[o:o + k]))


def test_adam_steps_reduce_the_loss(native, meshes):
    import torch
    from oracle import mpnn as M
    nbr, ew, dscale = face_graph(native, meshes, "pipe_small")
    n = len(nbr)
    rng = np.random.default_rng(9)
    v = rng.normal(size=n).astype(np.float32)
    # a target the network can approach: a smoothed copy of the input
    x = (v + M._aggregate(nbr, ew, v[:, None])[:, 0]).astype(np.float32)
    net = native.Mpnn(n, training=True)
    net.set_params(M.init_params(3))
    keep = [_dev(torch, nbr), _dev(torch, ew), _dev(torch, dscale)]
    g = net.graph(n, *keep)
    vd, xd = _dev(torch, v), _dev(torch, x)
    first = net.loss_backward(g, vd, xd)
    for step in range(1, 61):
        net.adam_step(2e-3, step)
        last = net.loss_backward(g, vd, xd)
    assert last < 0.7 * first, (first, last)


def test_backward_from_dz_matches_oracle(native, meshes):
    """nds_mpnn_backward (gradients from a given dL/dz, for losses evaluated
    outside the network) against the oracle's backward from the same dz."""
    import torch
    from oracle import mpnn as M
    nbr, ew, dscale = face_graph(native, meshes, "pipe_small")
    n = len(nbr)
    seg = [0, n // 3, n]
    rng = np.random.default_rng(11)
    v = rng.normal(size=n).astype(np.float32)
    dz = rng.normal(size=n).astype(np.float32)
    p = M.init_params(8)
    net = native.Mpnn(n, training=True)
    net.set_params(p)
    keep = [_dev(torch, nbr), _dev(torch, ew), _dev(torch, dscale)]
    g = net.graph(n, *keep)
    vd, dzd = _dev(torch, v), _dev(torch, dz)
    z = torch.zeros(n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    net.forward(g, vd, z, seg)
    net.backward(g, dzd)
    grads = net.grads()
    go, _ = M.grad_from_dz(p, nbr, ew, dscale, v, dz, seg)
    for l in (1, 2, 3):
        o = M.off_w(l)
        assert rel_l2(grads[o:o + 8192], go[o:o + 8192]) <= 2e-2, l
    assert rel_l2(grads[M.OFF_WD:M.OFF_WD + 66], go[M.OFF_WD:M.OFF_WD + 66]) <= 2e-2
    assert rel_l2(grads[:192], go[:192]) <= 2e-2
