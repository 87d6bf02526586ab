"""CPU restatement of the mixed-mesh pipe SIMPLE -- test infrastructure.

Follows the loop of the reference's HXT4B executable
(gpu/serial_cuda/hybrid_hxt4b/hxt4b_main.cu:236-258): per iteration the lagged
central advective convection of the current velocity (hex cells: the 27-point
Gauss rule over the Q1 + BF2 basis, hxt4b_main.cu:40-131 and
hybrid_hxt2/hxt2_main.cu:176-187; tet cells: the reference tensor
T[a][m][b][j] = int phi_a phi_m dphi_b/dxi_j), the relaxed rows and rAU,
the momentum right-hand sides, the multicolour Gauss-Seidel work (sgs1:
forward then backward colours), the continuity residual B u (zero at the
pin), a Jacobi-PCG pressure correction and p -= alpha_p dp.  Like the H8
oracle it consumes the product's host setup (velocity CSR pattern and its
constant values, gather lists, colours, divergence) through the C ABI
(nds_hybrid_flow_setup); the mesh comes from the HXT1 file itself.  Numpy,
small meshes only.
"""
from __future__ import annotations

import numpy as np

from oracle.hybrid_vtu import read_mixed_hxt1

_SIGN = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)
# face f of the reference hex: (normal axis, side) for z-, z+, y-, x+, y+, x-
_FACES = ((2, -1.0), (2, 1.0), (1, -1.0), (0, 1.0), (1, 1.0), (0, -1.0))


def hex_basis(x, y, z):
    """Q1 + BF2 values (14) and reference gradients (14 x 3) at one point."""
    phi, g = np.zeros(14), np.zeros((14, 3))
    c = np.array([x, y, z])
    for a in range(8):
        s = _SIGN[a]
        f = 1.0 + s * c
        phi[a] = 0.125 * f[0] * f[1] * f[2]
        g[a] = 0.125 * s * np.array([f[1] * f[2], f[0] * f[2], f[0] * f[1]])
    b, d = 1.0 - c * c, -2.0 * c
    for fi, (n, sg) in enumerate(_FACES):
        t1, t2 = (1 if n == 0 else 0), (1 if n == 2 else 2)
        s = 0.5 * (1.0 + sg * c[n])
        phi[8 + fi] = s * b[t1] * b[t2]
        g[8 + fi, n] = 0.5 * sg * b[t1] * b[t2]
        g[8 + fi, t1] = s * d[t1] * b[t2]
        g[8 + fi, t2] = s * b[t1] * d[t2]
    return phi, g


class HybridFlowOracle:
    def __init__(self, native, path, **opts):
        self.o = native.HybridFlowOptions.make(**opts)
        self.h = native.HybridAmg(path, None, options=self.o)
        a = self.h.array
        sc = a("flow.scalars")
        self.pin, self.nh, self.nt = int(sc[0]), int(sc[5]), int(sc[6])
        self.row, self.col, self.dpos = a("flow.row"), a("flow.col"), a("flow.diagPos")
        self.base, self.dr = a("flow.base"), a("flow.diagRBase")
        self.soff, self.src = a("flow.srcOff"), a("flow.src")
        self.fixed = a("flow.fixed").astype(bool)
        self.u = [a("flow.u0"), a("flow.u1"), a("flow.u2")]
        coff, crows = a("flow.colourOff"), a("flow.colourRows")
        self.colours = [crows[coff[c]:coff[c + 1]] for c in range(len(coff) - 1)]
        self.brow, self.bcol = a("b.row"), a("b.col")
        self.bx, self.by, self.bz = a("b.bx"), a("b.by"), a("b.bz")
        self.T = a("centT").reshape(8, 8, 8, 3)
        m = read_mixed_hxt1(path)
        self.m = m
        nv, npr = len(self.u[0]), self.nh + self.nt
        self.nv, self.np = nv, npr
        self.p = np.zeros(npr)
        # hex tables at the 27 points
        gx = np.array([-np.sqrt(0.6), 0.0, np.sqrt(0.6)])
        gw = np.array([5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0])
        self.qphi, self.qg, self.qw = [], [], []
        for ix in range(3):
            for iy in range(3):
                for iz in range(3):
                    ph, g = hex_basis(gx[ix], gx[iy], gx[iz])
                    self.qphi.append(ph)
                    self.qg.append(g)
                    self.qw.append(gw[ix] * gw[iy] * gw[iz])
        self.qphi, self.qg, self.qw = np.array(self.qphi), np.array(self.qg), np.array(self.qw)
        X = m["points"][m["hexes"]]  # (nh, 8, 3)
        J = np.einsum("cai,qaj->cqij", X, self.qg[:, :8, :])  # d x_i / d xi_j
        self.hdet = np.linalg.det(J)
        self.hinv = np.linalg.inv(J)  # [c, q, j, d] = d xi_j / d x_d
        # physical gradients of the 14 functions at each point: gp[c, q, a, d]
        self.hgp = np.einsum("qaj,cqjd->cqad", self.qg, self.hinv)
        self.hdofs, self.tdofs, self.tgeom = m["hex_dofs"], m["tet_dofs"], m["tet_geom"]

    def convection(self):
        u = np.stack(self.u, axis=1)  # (nv, 3)
        # hex blocks: C_ab = sum_q det w phi_a (u_q . grad phi_b)
        uh = u[self.hdofs]  # (nh, 14, 3)
        uq = np.einsum("qa,cad->cqd", self.qphi, uh)
        ug = np.einsum("cqd,cqbd->cqb", uq, self.hgp)
        dw = self.hdet * self.qw[None, :]
        hex_loc = np.einsum("cq,qa,cqb->cab", dw, self.qphi, ug).reshape(self.nh, 196)
        # tet blocks: C_ab = det sum_m sum_j (J^-1 u_m)_j T[a][m][b][j]
        ut = u[self.tdofs]  # (nt, 8, 3)
        I = self.tgeom[:, 3:12].reshape(-1, 3, 3)  # [t, j, d]
        ur = np.einsum("tmd,tjd->tmj", ut, I)
        tet_loc = np.einsum("tmj,ambj->tab", ur, self.T) * self.tgeom[:, 2][:, None, None]
        local = np.concatenate((hex_loc.ravel(), tet_loc.reshape(self.nt, 64).ravel()))
        conv = np.add.reduceat(local[self.src], self.soff[:-1]) if len(self.src) else np.zeros(len(self.col))
        empty = self.soff[1:] == self.soff[:-1]
        conv[empty] = 0.0
        return conv

    def _bmat(self, vals):
        import scipy.sparse as sp
        return sp.csr_matrix((vals, self.bcol, self.brow), shape=(self.np, self.nv))

    def step(self):
        o = self.o
        conv = self.convection()
        val = self.base + conv
        d = val[self.dpos].copy()
        dorig = d.copy()
        free = ~self.fixed
        den = self.dr + conv[self.dpos]
        rau = np.where(free, o.rau_scale * o.alpha_u / np.where(free, den, 1.0), 0.0)
        val[self.dpos[free]] = d[free] / o.alpha_u
        import scipy.sparse as sp
        A = sp.csr_matrix((val, self.col, self.row), shape=(self.nv, self.nv))
        Bx, By, Bz = self._bmat(self.bx), self._bmat(self.by), self._bmat(self.bz)
        bt = [Bx.T @ self.p, By.T @ self.p, Bz.T @ self.p]
        rhs = [np.where(free, bt[k] + ((1.0 - o.alpha_u) / o.alpha_u) * dorig * self.u[k], 0.0) for k in range(3)]
        diag = val[self.dpos]
        offd = A - sp.diags(diag)
        offd = offd.tocsr()
        orders = []
        if o.momentum_work == 0:
            orders = [self.colours]
        elif o.momentum_work == 1:
            orders = [self.colours if (self.it & 1) else self.colours[::-1]]
        else:
            orders = [self.colours, self.colours[::-1]]
        for k in range(3):
            x = self.u[k]
            for seq in orders:
                for rows in seq:
                    s = offd[rows] @ x
                    gs = (rhs[k][rows] - s) / diag[rows]
                    x[rows] = x[rows] + o.mom_omega * (gs - x[rows])
        cont = Bx @ self.u[0] + By @ self.u[1] + Bz @ self.u[2]
        cont[self.pin] = 0.0
        cn = float(np.sqrt(np.dot(cont, cont)))
        # Jacobi PCG on S = B diag(rau) B^T, pin row and column removed
        R = sp.diags(rau)
        S = (Bx @ R @ Bx.T + By @ R @ By.T + Bz @ R @ Bz.T).tocsr()
        sd = S.diagonal().copy()
        sd[self.pin] = 1.0
        inv = 1.0 / sd

        def Sop(v):
            w = v.copy()
            w[self.pin] = 0.0
            y = S @ w
            y[self.pin] = 0.0
            return y
        x = np.zeros(self.np)
        r = cont - Sop(x)
        r[self.pin] = 0.0
        r0 = float(np.sqrt(r @ r))
        its = 0
        if r0 > 0:
            target = max(o.p_atol, o.p_rtol * r0)
            z = inv * r
            z[self.pin] = 0.0
            pdir = z.copy()
            rho = r @ z
            for k in range(o.p_max):
                q = Sop(pdir)
                alpha = rho / (pdir @ q)
                x += alpha * pdir
                r -= alpha * q
                x[self.pin] = r[self.pin] = 0.0
                its = k + 1
                if np.sqrt(r @ r) <= target:
                    break
                z = inv * r
                z[self.pin] = 0.0
                nr = r @ z
                pdir = z + (nr / rho) * pdir
                pdir[self.pin] = 0.0
                rho = nr
        self.p = np.where(np.arange(self.np) == self.pin, 0.0, self.p - o.alpha_p * x)
        return cn, its

    def run(self, n):
        """relCont and pressure iterations of the first n iterations."""
        out = []
        c0 = None
        for self.it in range(1, n + 1):
            cn, its = self.step()
            c0 = cn if c0 is None else c0
            out.append((cn / max(c0, 1e-300), cn, its))
        return out
