"""CPU oracle of the learned pressure stage (test infrastructure only).

A numpy restatement of the network of nodals_b200/csrc/cuda/mpnn.cu -- there
is no reference counterpart, so this file is the definition the CUDA kernels
are checked against: forward values, the loss and every parameter gradient.
It rounds to BF16 (round to nearest even) at the same points as the kernels:
the encoder output h0 and every stored activation h^l, the aggregated
messages m^l that enter a dense layer, the dense layers' inputs, and the
back-propagated deltas that enter the tensor-core GEMMs.  Sums are float64
(the kernels accumulate in FP32 inside the tensor core and FP64 in the
reductions), so GPU and oracle agree to the rounding of a few BF16 values.

``exact=True`` drops every BF16 rounding: the network is then a smooth
function of its parameters (away from ReLU kinks) and ``grad`` can be checked
against central finite differences.
"""
from __future__ import annotations

import numpy as np

H = 64
NPARAM = 25026
OFF_WE, OFF_BE = 0, 128


def off_w(l):
    return 192 + (l - 1) * (H * 2 * H + H)


def off_b(l):
    return off_w(l) + H * 2 * H


OFF_WD = 192 + 3 * (H * 2 * H + H)
OFF_BD = OFF_WD + H
OFF_CS = OFF_BD + 1
assert OFF_CS + 1 == NPARAM


def bf16(x, exact=False):
    """Round float values to bfloat16 (nearest even), returned as float64."""
    if exact:
        return np.asarray(x, dtype=np.float64)
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounding = 0x7FFF + ((u >> 16) & 1)
    u = ((u + rounding) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return dict(We=p[OFF_WE:OFF_WE + 2 * H].reshape(H, 2), be=p[OFF_BE:OFF_BE + H],
                W=[p[off_w(l):off_w(l) + H * 2 * H].reshape(H, 2 * H) for l in (1, 2, 3)],
                b=[p[off_b(l):off_b(l) + H] for l in (1, 2, 3)],
                wd=p[OFF_WD:OFF_WD + H], bd=p[OFF_BD], cs=p[OFF_CS])


def init_params(seed=0):
    """He-style initial parameters (the training script's starting point)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM)
    p[OFF_WE:OFF_WE + 2 * H] = rng.normal(0, np.sqrt(2.0 / 2), 2 * H)
    for l in (1, 2, 3):
        p[off_w(l):off_w(l) + H * 2 * H] = rng.normal(0, np.sqrt(2.0 / (2 * H)), H * 2 * H)
    p[OFF_WD:OFF_WD + H] = rng.normal(0, np.sqrt(1.0 / H), H)
    p[OFF_CS] = 1.0
    return p.astype(np.float32)


def _aggregate(nbr, ew, h):
    m = np.zeros_like(h)
    for k in range(nbr.shape[1]):
        j = nbr[:, k]
        ok = j >= 0
        m[ok] += ew[ok, k][:, None] * h[j[ok]]
    return m


def _aggregate_t(nbr, ew, dm):
    """Transpose of _aggregate (the face graph and e are symmetric, so this
    equals _aggregate itself; written out for the oracle's own check)."""
    out = np.zeros_like(dm)
    for k in range(nbr.shape[1]):
        j = nbr[:, k]
        ok = j >= 0
        np.add.at(out, j[ok], ew[ok, k][:, None] * dm[ok])
    return out


def forward(p, nbr, ew, dscale, v, segs=None, exact=False):
    """z = N(v); returns z and the cache for backward.  nbr, ew: [n, 4];
    segs: offsets of independently normalised segments (default one)."""
    P = unpack(p)
    n = len(v)
    nbr = np.asarray(nbr).reshape(n, 4)
    ew = np.asarray(ew, dtype=np.float64).reshape(n, 4)
    v = np.asarray(v, dtype=np.float64)
    dscale = np.asarray(dscale, dtype=np.float64)
    segs = [0, n] if segs is None else list(segs)
    q = v * dscale
    sigma = np.ones(n)
    for a, b in zip(segs[:-1], segs[1:]):
        s = np.sqrt(np.mean(q[a:b] ** 2))
        sigma[a:b] = s if s > 0 else 1.0
    s = q / sigma
    f = np.stack([s, _aggregate(nbr, ew, s[:, None])[:, 0]], axis=1)
    pre0 = f @ P["We"].T + P["be"]
    h = [bf16(np.maximum(pre0, 0.0), exact)]
    X = []
    for l in range(3):
        m = _aggregate(nbr, ew, h[l])
        x = np.concatenate([h[l], bf16(m, exact)], axis=1)
        X.append(x)
        pre = x @ bf16(P["W"][l], exact).T + P["b"][l]
        h.append(bf16(np.maximum(pre, 0.0), exact))
    out = h[3] @ P["wd"] + P["bd"] + P["cs"] * s
    z = out * sigma * dscale  # sigma out / sqrt(a_ii)
    cache = dict(P=P, nbr=nbr, ew=ew, f=f, s=s, h=h, X=X, out=out, sigma=sigma, dscale=dscale, segs=segs,
                 pre0=pre0, exact=exact)
    return z, cache


def loss_grad(p, nbr, ew, dscale, v, x, segs=None, exact=False):
    """Loss (mean over segments of sum (out - t)^2 / sum t^2, t = x / (dscale
    sigma)) and its gradient in the parameter layout."""
    z, c = forward(p, nbr, ew, dscale, v, segs, exact)
    P, nbr, ew, segs = c["P"], c["nbr"], c["ew"], c["segs"]
    n = len(v)
    t = np.asarray(x, dtype=np.float64) / (c["dscale"] * c["sigma"])
    d = c["out"] - t
    nseg = len(segs) - 1
    loss = 0.0
    dout = np.zeros(n)
    for a, b in zip(segs[:-1], segs[1:]):
        tt = max(np.sum(t[a:b] ** 2), 1e-300)
        loss += np.sum(d[a:b] ** 2) / tt / nseg
        dout[a:b] = 2.0 * d[a:b] / (tt * nseg)
    return loss, _backward(c, dout), c


def grad_from_dz(p, nbr, ew, dscale, v, dz, segs=None, exact=False):
    """Parameter gradient of sum_i dz_i z_i (z = N(v)), i.e. the backward
    pass from a given dL/dz: dout = dz sigma dscale."""
    z, c = forward(p, nbr, ew, dscale, v, segs, exact)
    return _backward(c, np.asarray(dz, dtype=np.float64) * c["sigma"] * c["dscale"]), c


def _backward(c, dout):
    P, nbr, ew = c["P"], c["nbr"], c["ew"]
    g = np.zeros(NPARAM)
    h, X = c["h"], c["X"]
    g[OFF_WD:OFF_WD + H] = dout @ h[3]
    g[OFF_BD] = dout.sum()
    g[OFF_CS] = dout @ c["s"]
    dh = np.outer(dout, P["wd"])
    for l in (3, 2, 1):
        delta = bf16(dh * (h[l] > 0), c["exact"])
        g[off_w(l):off_w(l) + H * 2 * H] = (delta.T @ X[l - 1]).ravel()
        g[off_b(l):off_b(l) + H] = delta.sum(axis=0)
        dX = delta @ bf16(P["W"][l - 1], c["exact"])
        dh = dX[:, :H] + _aggregate_t(nbr, ew, dX[:, H:])
    delta0 = dh * (c["pre0"] > 0)
    g[OFF_WE:OFF_WE + 2 * H] = (delta0.T @ c["f"]).ravel()
    g[OFF_BE:OFF_BE + H] = delta0.sum(axis=0)
    return g
