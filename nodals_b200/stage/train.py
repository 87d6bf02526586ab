"""Training of the learned pressure stage on one GPU.

The stage z = N(b) acts ahead of the V-cycle inside FGMRES, where it is kept
only when it reduces the residual (||b - A z|| < ||b||).  It is trained for
exactly that, on the live operators of the plain solver:

* a pool of POOL members of the seeded pipe family (``meshgen.family_member``:
  64 training and 16 held-out pipes of ~200k tets, radius, length, bend angle
  and Re drawn from their seeds), each a running mixed-precision AMG-PCG
  solver; every training step advances each member by 1-4 SIMPLE iterations
  and takes its latest pressure-correction pair (b, x = A^-1 b) with the face
  graph, edge weights and scaling of that iteration's operator
  (``nds_solver_pressure_pair``, ``nds_solver_stage_graph``); every
  SWAP_EVERY steps the oldest member is replaced by the next training pipe;
* the batch is the POOL graphs joined as one graph of POOL segments (each
  normalised on its own); the network (this package's tcgen05 kernels)
  computes z = N(b);
* per segment, with the operator A of that solver and D = diag(A), the loss
  is the Jacobi-scaled residual ||D^-1/2 (b - A z)||^2 / ||D^-1/2 b||^2 plus
  SUP times the diagonal-weighted error against the solver's own solution,
  sum D (z - x)^2 / sum D x^2; dL/dz = -2 A D^-1 (b - A z) / ||D^-1/2 b||^2
  + SUP 2 D (z - x) / sum D x^2 needs two products with A
  (``nds_solver_apply_operator``); ``nds_mpnn_backward`` takes it from there,
  then Adam (``nds_mpnn_adam_step``).

    python -m nodals_b200.stage.train --out nodals_b200/stage/mpnn_params.bin --log train_log.json
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .. import meshgen
from .. import native as N

SOLVER = dict(alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, run_mode="converge", simple_tol=1e-12,
              max_outer=1000000, amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg",
              precision="mixed", p_krylov="pcg", geom_from_inlet=1, amg_terminal=300)
POOL, SWAP_EVERY, SUP = 8, 20, 0.1


class Member:
    """A running solver of one family member."""

    def __init__(self, index: int, torch, warm: int = 3):
        tm, re, prm = meshgen.family_member(index)
        self.index, self.prm = index, prm
        self.P = N.Problem(N.Mesh.from_tetmesh(tm), re=re, **SOLVER)
        self.S = N.Solver(self.P)
        self.n = self.S.nc
        self.nbr = torch.empty(4 * self.n, dtype=torch.int32, device="cuda")
        for _ in range(warm):
            self.S.step()
        torch.cuda.synchronize()
        N.solver_stage_graph(self.S, self.nbr, None, None)

    def advance(self, k: int):
        for _ in range(k):
            self.S.step()

    def sample(self, ew, ds, b, x):
        N.solver_stage_graph(self.S, None, ew, ds)
        N.solver_pressure_pair(self.S, b, x)


def residual_loss(members, z, b, x, ds, segs, torch, grad=True):
    """Mean over segments of the scaled residual (+ SUP x the weighted error)
    and dL/dz (device)."""
    dz = torch.zeros_like(z) if grad else None
    tmp = torch.empty_like(z)
    losses = []
    nseg = len(members)
    for i, m in enumerate(members):
        a, e = segs[i], segs[i + 1]
        zs, bs, xs, dsi = z[a:e], b[a:e], x[a:e], ds[a:e]
        torch.cuda.synchronize()
        N.solver_apply_operator(m.S, zs, tmp[a:e])
        torch.cuda.synchronize()
        r = bs - tmp[a:e]
        d = dsi * dsi                     # 1 / a_ii
        bb = float(torch.sum(d * bs * bs))
        w = 1.0 / (dsi * dsi)             # a_ii
        xx = float(torch.sum(w * xs * xs))
        lres = float(torch.sum(d * r * r)) / bb
        lsup = float(torch.sum(w * (zs - xs) ** 2)) / xx
        losses.append((lres, lsup))
        if grad:
            q = (d * r).contiguous()
            torch.cuda.synchronize()
            N.solver_apply_operator(m.S, q, tmp[a:e])
            torch.cuda.synchronize()
            dz[a:e] = (-2.0 / bb) * tmp[a:e] + (SUP * 2.0 / xx) * w * (zs - xs)
    dz = None if dz is None else dz / nseg
    return float(np.mean([l[0] + SUP * l[1] for l in losses])), [l[0] for l in losses], dz


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--log")
    ap.add_argument("--steps", type=int, default=1200)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ns = ap.parse_args()
    import torch
    from . import init_params

    t0 = time.perf_counter()
    rng = np.random.default_rng(ns.seed)
    train_ids = list(range(meshgen.FAMILY_TRAIN))
    held_ids = list(range(meshgen.FAMILY_TRAIN, meshgen.FAMILY_TRAIN + 4))
    pool = [Member(i, torch, warm=3 + 5 * k) for k, i in enumerate(train_ids[:POOL])]
    nxt = POOL
    held = [Member(i, torch, warm=20) for i in held_ids]
    n = pool[0].n
    assert all(m.n == n for m in pool + held), "family members share one cell count"
    total = POOL * n
    segs = [k * n for k in range(POOL + 1)]
    net = N.Mpnn(total, training=True)
    net.set_params(init_params(ns.seed))
    f32 = dict(dtype=torch.float32, device="cuda")
    ew, ds, b, x, z = (torch.empty(4 * total, **f32), torch.empty(total, **f32), torch.empty(total, **f32),
                       torch.empty(total, **f32), torch.empty(total, **f32))
    nbr = torch.empty(4 * total, dtype=torch.int32, device="cuda")

    def join_graph(members):
        for k, m in enumerate(members):
            nbr[4 * k * n:4 * (k + 1) * n] = torch.where(m.nbr >= 0, m.nbr + k * n, m.nbr)
        torch.cuda.synchronize()

    def fill(members):
        torch.cuda.synchronize()
        for k, m in enumerate(members):
            m.sample(ew[4 * k * n:4 * (k + 1) * n], ds[k * n:(k + 1) * n], b[k * n:(k + 1) * n], x[k * n:(k + 1) * n])

    hn = len(held) * n
    hsegs = [k * n for k in range(len(held) + 1)]

    def held_loss():
        join_graph(held)
        fill(held)
        g = net.graph(hn, nbr[:4 * hn], ew[:4 * hn], ds[:hn])
        net.forward(g, b[:hn], z[:hn], hsegs)
        torch.cuda.synchronize()
        loss, per, _ = residual_loss(held, z[:hn], b[:hn], x[:hn], ds[:hn], hsegs, torch, grad=False)
        join_graph(pool)
        return per

    log = {"steps": [], "train_loss": [], "held_residual": [], "lr": ns.lr, "pool": POOL, "swap_every": SWAP_EVERY,
           "sup_weight": SUP, "members_used": []}
    log["held_residual_initial"] = held_loss()
    print("initial held-out scaled residuals", [round(v, 4) for v in log["held_residual_initial"]], flush=True)
    join_graph(pool)
    t1 = time.perf_counter()
    for step in range(1, ns.steps + 1):
        if step % SWAP_EVERY == 0:
            old = step // SWAP_EVERY % POOL
            pool[old] = Member(train_ids[nxt % len(train_ids)], torch, warm=3 + int(rng.integers(40)))
            log["members_used"].append(train_ids[nxt % len(train_ids)])
            nxt += 1
            join_graph(pool)
        for m in pool:
            m.advance(1 + int(rng.integers(4)))
        fill(pool)
        g = net.graph(total, nbr, ew, ds)
        net.forward(g, b, z, segs)
        torch.cuda.synchronize()
        loss, _, dz = residual_loss(pool, z, b, x, ds, segs, torch)
        torch.cuda.synchronize()
        net.backward(g, dz)
        lr = ns.lr * 0.5 * (1.0 + np.cos(np.pi * (step - 1) / ns.steps))
        net.adam_step(lr, step)
        if step % 100 == 0 or step == ns.steps:
            hl = held_loss()
            log["steps"].append(step)
            log["train_loss"].append(loss)
            log["held_residual"].append(hl)
            print(f"step {step}: train {loss:.4f} held-out residual {np.mean(hl):.4f} "
                  f"({time.perf_counter() - t1:.1f} s)", flush=True)
    log["train_seconds"] = time.perf_counter() - t1
    log["setup_seconds"] = t1 - t0
    net.params().tofile(ns.out)
    if ns.log:
        with open(ns.log, "w") as f:
            json.dump(log, f, indent=1)
    print("wrote", ns.out, flush=True)


if __name__ == "__main__":
    main()
