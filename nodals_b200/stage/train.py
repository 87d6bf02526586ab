"""Training of the learned pressure stage on one GPU.

1. Harvest.  For every member of the seeded pipe family
   (``meshgen.family_member``: 64 training and 16 held-out pipes of ~200k
   tets, radius, length, bend angle and Re drawn from their seeds) the plain
   mixed-precision AMG-PCG solver runs SIMPLE iterations; at the iterations
   in HARVEST the pressure-correction right-hand side b and solution x
   (``nds_solver_pressure_pair``) and the face graph with the edge weights
   and scaling of that iteration's operator (``nds_solver_stage_graph``) stay
   on the device.
2. Train.  Adam on batches of 8 pairs from 8 different training meshes,
   joined as one graph of 8 segments (each normalised on its own), with this
   package's forward, backward and Adam kernels (``nds_mpnn_*``).
3. Write the parameters (float32) and a JSON log of the losses.

    python -m nodals_b200.stage.train --out nodals_b200/stage/mpnn_params.bin --log train_log.json
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .. import meshgen
from .. import native as N

HARVEST = (3, 6, 10, 15, 20, 30, 40, 55, 70, 85, 100, 120)
SOLVER = dict(alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, run_mode="converge", simple_tol=1e-12,
              max_outer=100000, amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg",
              precision="mixed", p_krylov="pcg", geom_from_inlet=1, amg_terminal=300)


def harvest(index: int, torch, iters=HARVEST):
    """Graph (nbr) and per-iteration samples (ew, dscale, b, x) of one member."""
    tm, re, prm = meshgen.family_member(index)
    P = N.Problem(N.Mesh.from_tetmesh(tm), re=re, **SOLVER)
    S = N.Solver(P)
    n = S.nc
    nbr = torch.empty(4 * n, dtype=torch.int32, device="cuda")
    samples = []
    for it in range(1, max(iters) + 1):
        S.step()
        if it in iters:
            ew = torch.empty(4 * n, dtype=torch.float32, device="cuda")
            ds = torch.empty(n, dtype=torch.float32, device="cuda")
            b = torch.empty(n, dtype=torch.float32, device="cuda")
            x = torch.empty(n, dtype=torch.float32, device="cuda")
            N.solver_stage_graph(S, nbr if not samples else None, ew, ds)
            N.solver_pressure_pair(S, b, x)
            samples.append(dict(ew=ew, ds=ds, b=b, x=x, it=it))
    torch.cuda.synchronize()
    return dict(index=index, n=n, nbr=nbr, samples=samples, prm=prm)


def batch(members, picks, torch):
    """One graph of len(picks) segments: (member, sample) pairs joined."""
    nbrs, ews, dss, bs, xs, segs = [], [], [], [], [], [0]
    for mi, si in picks:
        m = members[mi]
        s = m["samples"][si]
        off = segs[-1]
        nb = m["nbr"]
        nbrs.append(torch.where(nb >= 0, nb + off, nb))
        ews.append(s["ew"])
        dss.append(s["ds"])
        bs.append(s["b"])
        xs.append(s["x"])
        segs.append(off + m["n"])
    return (torch.cat(nbrs), torch.cat(ews), torch.cat(dss), torch.cat(bs), torch.cat(xs), segs)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--log")
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--train", type=int, default=meshgen.FAMILY_TRAIN)
    ap.add_argument("--held-out", type=int, default=meshgen.FAMILY_HELD_OUT)
    ap.add_argument("--seed", type=int, default=0)
    ns = ap.parse_args()
    import torch
    from . import init_params

    t0 = time.perf_counter()
    members = []
    for i in range(ns.train + ns.held_out):
        members.append(harvest(i, torch))
        print(f"harvested member {i}: {members[-1]['n']} cells, {len(members[-1]['samples'])} pairs, "
              f"{time.perf_counter() - t0:.1f} s", flush=True)
    train_ids = list(range(ns.train))
    held_ids = list(range(ns.train, ns.train + ns.held_out))
    nmax = max(sum(sorted((members[i]["n"] for i in train_ids), reverse=True)[:ns.batch]),
               sum(members[i]["n"] for i in held_ids[:ns.batch]))
    net = N.Mpnn(nmax, training=True)
    net.set_params(init_params(ns.seed))
    rng = np.random.default_rng(ns.seed)
    nsamp = len(HARVEST)

    def run(ids, picks_rng, step=False):
        mids = picks_rng.choice(ids, size=min(ns.batch, len(ids)), replace=False)
        picks = [(int(m), int(picks_rng.integers(nsamp))) for m in mids]
        nbr, ew, ds, b, x, segs = batch(members, picks, torch)
        g = net.graph(len(b), nbr, ew, ds)
        return net.loss_backward(g, b, x, segs)

    def held_loss():
        r = np.random.default_rng(12345)
        return float(np.mean([run(held_ids, r) for _ in range(4)]))

    log = {"steps": [], "train_loss": [], "held_loss": [], "lr": ns.lr, "batch": ns.batch,
           "harvest_iterations": list(HARVEST), "members": [m["prm"] for m in members]}
    h0 = held_loss()
    log["held_loss_initial"] = h0
    print(f"initial held-out loss {h0:.4f}", flush=True)
    t1 = time.perf_counter()
    for step in range(1, ns.steps + 1):
        loss = run(train_ids, rng)
        lr = ns.lr * 0.5 * (1.0 + np.cos(np.pi * (step - 1) / ns.steps))
        net.adam_step(lr, step)
        if step % 100 == 0 or step == ns.steps:
            hl = held_loss()
            log["steps"].append(step)
            log["train_loss"].append(loss)
            log["held_loss"].append(hl)
            print(f"step {step}: train {loss:.4f} held-out {hl:.4f} ({time.perf_counter() - t1:.1f} s)", flush=True)
    log["train_seconds"] = time.perf_counter() - t1
    log["harvest_seconds"] = t1 - t0
    net.params().tofile(ns.out)
    if ns.log:
        with open(ns.log, "w") as f:
            json.dump(log, f, indent=1)
    print("wrote", ns.out, flush=True)


if __name__ == "__main__":
    main()
