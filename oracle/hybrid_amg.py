"""CPU restatement of the mixed-mesh pressure V-cycle -- test infrastructure.

Follows hxt4c::HybridAMG of the reference (gpu/serial_cuda/hybrid_hxt5b/
hybrid_amg.cuh): the zero-guess smoothers of smooth_zero (:445-487: damped
Jacobi, l1-Jacobi, the symmetric Chebyshev on D^-1/2 A D^-1/2 with roots of
cheb_root :400-403) and of mcgs (:405-433, colours from build_color
:195-215), the recursive vcycle (:500-517) and apply (:519-533).  Every work
vector is passed as the reference passes it, so the post-smoothing calls,
which hand one vector as both x and corr (and on the fine level as both b and
r), compute what the reference computes.  Numpy arrays stand in for the
device buffers; in-place updates keep that aliasing.  ``separate_post``
gives the post-smoothing calls work vectors of their own instead (the
product's symmetric variant).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp


def _csr(row, col, val, n, m):
    return sp.csr_matrix((np.asarray(val, dtype=np.float64), np.asarray(col), np.asarray(row)), shape=(n, m))


def colours(A: sp.csr_matrix):
    """Greedy colours: each row takes the smallest colour not held by a
    lower-numbered neighbour; rows of each colour ascending."""
    n = A.shape[0]
    col = np.full(n, -1)
    for i in range(n):
        nb = A.indices[A.indptr[i]:A.indptr[i + 1]]
        used = {int(col[j]) for j in nb if j < i}
        c = 0
        while c in used:
            c += 1
        col[i] = c
    return [np.flatnonzero(col == c) for c in range(int(col.max()) + 1)]


class Level:
    def __init__(self, A: sp.csr_matrix, colour: bool):
        self.A = A
        self.n = A.shape[0]
        self.d = A.diagonal().copy()
        self.l1 = np.asarray(abs(A).sum(axis=1)).ravel()
        self.b, self.x, self.r, self.tmp, self.corr = (np.zeros(self.n) for _ in range(5))
        self.colours = colours(A) if colour else None


class VCycle:
    """``arrays``: pressure matrix ``fine.*`` and hierarchy ``amg.*`` arrays as
    the reference's builders write them; ``opt``: smoother, cheb_degree,
    low_fraction, jacobi_omega, jacobi_fine/coarse_sweeps, mcgs_omega,
    mcgs_fine/coarse_sweeps."""

    def __init__(self, arrays: dict, opt: dict):
        self.o = dict(smoother="cheb2", cheb_degree=4, low_fraction=0.05, jacobi_omega=0.7, jacobi_fine_sweeps=1,
                      jacobi_coarse_sweeps=1, mcgs_omega=1.0, mcgs_fine_sweeps=1, mcgs_coarse_sweeps=1,
                      separate_post=False)
        self.o.update(opt)
        mc = self.o["smoother"] == "mcgs"
        n = len(arrays["fine.diag"])
        self.F = Level(_csr(arrays["fine.row"], arrays["fine.col"], arrays["fine.val"], n, n), mc)
        nlev = int(arrays["amg.levels"][0])
        self.L, self.P = [], []
        nf = n
        for l in range(nlev):
            nc = int(arrays[f"amg.P{l}.nCoarse"][0])
            self.P.append(_csr(arrays[f"amg.P{l}.row"], arrays[f"amg.P{l}.col"], arrays[f"amg.P{l}.val"], nf, nc))
            A = _csr(arrays[f"amg.A{l}.row"], arrays[f"amg.A{l}.col"], arrays[f"amg.A{l}.val"], nc, nc)
            self.L.append(Level(A, mc and l + 1 < nlev))
            nf = nc
        tn = self.L[-1].n
        self.inv = np.asarray(arrays["amg.terminal_inv"], dtype=np.float64).reshape(tn, tn)
        self.fine_lambda = float(arrays["amg.fineLambda"][0])
        self.level_lambda = np.asarray(arrays["amg.levelLambda"], dtype=np.float64)

    @staticmethod
    def cheb_root(hi, lo, k, degree):
        centre, radius = 0.5 * (hi + lo), 0.5 * (hi - lo)
        return centre - radius * math.cos(math.pi * (2.0 * k + 1.0) / (2.0 * degree))

    def smooth(self, lev: Level, b, x, tmp, r, corr, sweeps, lam):
        o, A, sq = self.o, lev.A, np.sqrt(lev.d)
        if o["smoother"] == "mcgs":
            x[:] = 0.0
            w = o["mcgs_omega"]
            for _ in range(sweeps):
                for cols in (lev.colours, lev.colours[::-1]):
                    for rows in cols:
                        for i in rows:
                            lo_, hi_ = A.indptr[i], A.indptr[i + 1]
                            js, vs = A.indices[lo_:hi_], A.data[lo_:hi_]
                            off = float(np.dot(vs[js != i], x[js[js != i]]))
                            old = x[i]
                            x[i] = old + w * ((b[i] - off) / lev.d[i] - old)
            return
        if o["smoother"] in ("jacobi", "l1jacobi"):
            den = lev.l1 if o["smoother"] == "l1jacobi" else lev.d
            w = o["jacobi_omega"]
            x[:] = w * b / den
            for _ in range(1, sweeps):
                tmp[:] = A @ x
                r[:] = b - tmp
                x[:] = x + w * r / den
            return
        lo = o["low_fraction"] * lam
        if not (lam > lo > 0):
            raise ValueError("Chebyshev interval invalid")
        deg = o["cheb_degree"]
        r[:] = b / sq
        x[:] = (1.0 / self.cheb_root(lam, lo, 0, deg)) * r
        for k in range(1, deg):
            tmp[:] = x / sq
            corr[:] = A @ tmp
            corr[:] = corr / sq
            x[:] = x + (1.0 / self.cheb_root(lam, lo, k, deg)) * (r - corr)
        x[:] = x / sq

    def _sweeps(self, fine):
        o = self.o
        if o["smoother"] == "mcgs":
            return o["mcgs_fine_sweeps"] if fine else o["mcgs_coarse_sweeps"]
        return o["jacobi_fine_sweeps"] if fine else o["jacobi_coarse_sweeps"]

    def _work(self, lev, post):
        if post and self.o["separate_post"]:
            return np.zeros(lev.n), np.zeros(lev.n)
        return lev.r, lev.corr

    def smooth_fine(self, b, x, post=False):
        F = self.F
        r, corr = self._work(F, post)
        self.smooth(F, b, x, F.tmp, r, corr, self._sweeps(True), self.fine_lambda)

    def smooth_coarse(self, l, b, x, post=False):
        A = self.L[l]
        lam = float(self.level_lambda[l]) if l < len(self.level_lambda) else 0.0
        r, corr = self._work(A, post)
        self.smooth(A, b, x, A.tmp, r, corr, self._sweeps(False), lam)

    def vcycle(self, l, b, x):
        A = self.L[l]
        if l + 1 == len(self.L):
            x[:] = self.inv @ b
            return
        self.smooth_coarse(l, b, x)
        A.tmp[:] = A.A @ x
        A.r[:] = b - A.tmp
        C = self.L[l + 1]
        C.b[:] = self.P[l + 1].T @ A.r
        self.vcycle(l + 1, C.b, C.x)
        x[:] = x + self.P[l + 1] @ C.x
        A.tmp[:] = A.A @ x
        A.r[:] = b - A.tmp
        A.b[:] = A.r
        self.smooth_coarse(l, A.b, A.corr, post=True)
        x[:] = x + A.corr

    def apply(self, b) -> np.ndarray:
        F = self.F
        b = np.asarray(b, dtype=np.float64)
        z = np.zeros(F.n)
        self.smooth_fine(b, z)
        F.tmp[:] = F.A @ z
        F.r[:] = b - F.tmp
        C = self.L[0]
        C.b[:] = self.P[0].T @ F.r
        self.vcycle(0, C.b, C.x)
        z[:] = z + self.P[0] @ C.x
        F.tmp[:] = F.A @ z
        F.r[:] = b - F.tmp
        self.smooth_fine(F.r, F.corr, post=True)
        z[:] = z + F.corr
        return z
