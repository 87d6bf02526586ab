"""The learned stage's CPU oracle (oracle/mpnn.py) against itself: its
backward pass against central finite differences of its own loss with the
BF16 roundings off (the network is then smooth away from ReLU kinks), and
the transpose of the neighbour aggregation against the aggregation (the
face graph and its edge weights are symmetric)."""
from __future__ import annotations

import numpy as np

from oracle import mpnn as M


def small_graph(n=40, seed=1):
    """A symmetric graph with at most four neighbours per node (a ring with
    chords), symmetric positive edge weights and a positive scaling."""
    rng = np.random.default_rng(seed)
    nbr = -np.ones((n, 4), dtype=np.int32)
    cnt = np.zeros(n, dtype=int)
    w = {}

    def add(a, b, e):
        if a == b or cnt[a] >= 4 or cnt[b] >= 4 or (a, b) in w:
            return
        nbr[a, cnt[a]] = b
        nbr[b, cnt[b]] = a
        cnt[a] += 1
        cnt[b] += 1
        w[(a, b)] = w[(b, a)] = e

    for i in range(n):
        add(i, (i + 1) % n, -0.2 - 0.1 * rng.random())
    for i in range(0, n, 3):
        add(i, (i + 7) % n, -0.15 * rng.random())
    ew = np.zeros((n, 4))
    for i in range(n):
        for k in range(4):
            if nbr[i, k] >= 0:
                ew[i, k] = w[(i, nbr[i, k])]
    dscale = 0.5 + rng.random(n)
    return nbr, ew, dscale


def test_aggregate_transpose_is_the_aggregate():
    nbr, ew, _ = small_graph()
    x = np.random.default_rng(0).normal(size=(len(nbr), 5))
    assert np.allclose(M._aggregate(nbr, ew, x), M._aggregate_t(nbr, ew, x))


def test_oracle_gradient_against_finite_differences():
    nbr, ew, dscale = small_graph()
    n = len(nbr)
    rng = np.random.default_rng(3)
    v = rng.normal(size=n)
    x = rng.normal(size=n)
    p = M.init_params(5).astype(np.float64)
    segs = [0, 17, n]
    _, g, _ = M.loss_grad(p, nbr, ew, dscale, v, x, segs, exact=True)
    # a sample of every parameter block
    idx = list(range(0, 128, 9)) + list(range(128, 192, 7))
    for l in (1, 2, 3):
        idx += list(range(M.off_w(l), M.off_w(l) + 8192, 613)) + list(range(M.off_b(l), M.off_b(l) + 64, 11))
    idx += list(range(M.OFF_WD, M.OFF_WD + 64, 5)) + [M.OFF_BD, M.OFF_CS]
    eps = 1e-6
    for i in idx:
        a, b = p.copy(), p.copy()
        a[i] += eps
        b[i] -= eps
        la, _, _ = M.loss_grad(a, nbr, ew, dscale, v, x, segs, exact=True)
        lb, _, _ = M.loss_grad(b, nbr, ew, dscale, v, x, segs, exact=True)
        fd = (la - lb) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.005859375, -3.1415926, 1e-20, 65504.0], dtype=np.float32)
    r = M.bf16(vals)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to even -> 1
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125)
    assert abs(r[3] - (-3.140625)) < 1e-12
