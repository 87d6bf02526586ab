"""ctypes driver of the C oracle (oracle/h8_oracle.c) -- test infrastructure.

``Oracle(problem)`` takes a ``nodals_b200.native.Problem`` (host setup whose
arrays are pinned against the reference's own setup builders) and runs the
FP64 CPU restatement of the reference SIMPLE loop on it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_P = C.POINTER


class _Level(C.Structure):
    _fields_ = [("n", C.c_int), ("row", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p), ("diag", C.c_void_p)]


class _Xfer(C.Structure):
    _fields_ = [("nf", C.c_int), ("nc", C.c_int), ("row", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p)]


_PTRS = ["mrow", "mcol", "K", "mdpos", "color_off", "color_rows", "inc_off", "inc", "ref", "row_slot", "det", "invJ",
         "bco", "fixed", "fixed_div", "s0", "s1", "s2", "centT", "init_rau", "frow", "fcol", "fdpos", "fcontrib_off",
         "fslot"]


class _Problem(C.Structure):
    _fields_ = ([("nc", C.c_int), ("nv", C.c_int), ("ncolors", C.c_int)] + [(n, C.c_void_p) for n in _PTRS] +
                [("nlev", C.c_int), ("L", C.c_void_p), ("P", C.c_void_p), ("tinv", C.c_void_p), ("power_its", C.c_int),
                 ("alpha_u", C.c_double), ("alpha_p", C.c_double), ("rau_scale", C.c_double),
                 ("simple_tol", C.c_double), ("mom_omega", C.c_double),
                 ("run_mode", C.c_int), ("momentum_work", C.c_int), ("pressure_solver", C.c_int),
                 ("p_rtol", C.c_double), ("p_atol", C.c_double), ("p_max", C.c_int),
                 ("p_richardson_omega", C.c_double), ("p_cheb_degree", C.c_int), ("p_power_its", C.c_int),
                 ("p_cheb_low_fraction", C.c_double), ("p_power_safety", C.c_double),
                 ("amg_smoother", C.c_int), ("amg_cheb_degree", C.c_int),
                 ("amg_lambda_safety", C.c_double), ("amg_lambda_low_fraction", C.c_double),
                 ("amg_jacobi_omega", C.c_double), ("amg_jacobi_fine_sweeps", C.c_int),
                 ("amg_jacobi_coarse_sweeps", C.c_int), ("threads", C.c_int),
                 ("supg", C.c_int), ("nu", C.c_double), ("supg_tau_scale", C.c_double), ("supg_magic", C.c_double),
                 ("h2", C.c_void_p), ("supg_rule", C.c_void_p)])


class Report(C.Structure):
    _fields_ = [("it", C.c_int), ("rel_cont", C.c_double), ("cont_norm", C.c_double), ("p_its", C.c_int),
                ("p_rel", C.c_double), ("p_ok", C.c_int), ("audited", C.c_int), ("audit_rel", C.c_double * 3),
                ("converged", C.c_int), ("status", C.c_int), ("ms_total", C.c_double), ("ms_pressure", C.c_double)]


_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.ora_create.restype = C.c_void_p
        L.ora_create.argtypes = [C.c_void_p]
        L.ora_step.argtypes = [C.c_void_p, C.POINTER(Report)]
        L.ora_get.argtypes = [C.c_void_p] * 5
        L.ora_set.argtypes = [C.c_void_p] * 5
        L.ora_fine_lambda.restype = C.c_double
        L.ora_fine_lambda.argtypes = [C.c_void_p]
        L.ora_destroy.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Oracle:
    def __init__(self, problem, threads: int = 0):
        o = problem.options
        if o.amg_smoother == 3:
            raise NotImplementedError("the oracle restates cheb2, jacobi and l1jacobi smoothers")
        self._keep = {}

        def arr(name, dtype=None):
            a = problem.array(name)
            if dtype is not None:
                a = a.astype(dtype)
            a = np.ascontiguousarray(a)
            self._keep[name + str(dtype)] = a
            return a

        from nodals_b200.native import lib as _nl  # noqa: F401  (problem already built)
        cent = np.ascontiguousarray(problem.array("centT"))
        self._keep["centT"] = cent
        P = _Problem()
        c = problem.counts()
        P.nc, P.nv, P.ncolors = c["nc"], c["nv"], c["ncolors"]
        src = {"mrow": ("mom.row", None), "mcol": ("mom.col", None), "K": ("mom.val", None),
               "mdpos": ("mom.diagPos", None), "color_off": ("color.offset", None), "color_rows": ("color.rows", None),
               "inc_off": ("fine.incOff", None), "inc": ("fine.packed", None), "ref": ("cell.ref", None),
               "row_slot": ("cell.rowSlot", None), "det": ("cell.det", None), "invJ": ("cell.invJ", None),
               "bco": ("cell.bcoeff", None), "fixed": ("fixedValue", None), "fixed_div": ("fixedDiv", None),
               "s0": ("staticRhs0", None), "s1": ("staticRhs1", None), "s2": ("staticRhs2", None),
               "init_rau": ("initRau", None), "frow": ("fine.row", None), "fcol": ("fine.col", None),
               "fdpos": ("fine.diagPos", None), "fcontrib_off": ("fine.contribOff", None), "fslot": ("fine.slot", None)}
        for f, (name, dt) in src.items():
            setattr(P, f, _ptr(arr(name, dt)))
        P.centT = _ptr(cent)
        nlev = int(problem.scalar("amg.levels"))
        levels = (_Level * nlev)()
        xfers = (_Xfer * nlev)()
        for l in range(nlev):
            row, col, val, dg = (arr(f"amg.A{l}.{k}") for k in ("row", "col", "val", "diag"))
            levels[l] = _Level(len(dg), _ptr(row), _ptr(col), _ptr(val), _ptr(dg))
            prow, pcol, pval = (arr(f"amg.P{l}.{k}") for k in ("row", "col", "val"))
            xfers[l] = _Xfer(len(prow) - 1, int(problem.scalar(f"amg.P{l}.nCoarse")), _ptr(prow), _ptr(pcol), _ptr(pval))
        self._keep["levels"], self._keep["xfers"] = levels, xfers
        P.nlev = nlev
        P.L = C.addressof(levels)
        P.P = C.addressof(xfers)
        P.tinv = _ptr(arr("amg.terminal_inv"))
        P.power_its = int(problem.scalar("amg.powerIts"))
        for k in ("alpha_u", "alpha_p", "rau_scale", "simple_tol", "mom_omega", "run_mode", "momentum_work",
                  "pressure_solver", "p_rtol", "p_atol", "p_max", "p_richardson_omega", "p_cheb_degree", "p_power_its",
                  "p_cheb_low_fraction", "p_power_safety", "amg_smoother", "amg_cheb_degree", "amg_lambda_safety",
                  "amg_lambda_low_fraction", "amg_jacobi_omega", "amg_jacobi_fine_sweeps", "amg_jacobi_coarse_sweeps"):
            setattr(P, k, getattr(o, k))
        P.threads = threads
        P.supg = o.supg
        P.nu = problem.scalar("pipe.nu")
        P.supg_tau_scale, P.supg_magic = o.supg_tau_scale, o.supg_magic
        P.h2 = _ptr(arr("cell.h2"))
        P.supg_rule = _ptr(arr("supg.rule"))
        self._P = P
        self.nc, self.nv = P.nc, P.nv
        self._h = lib().ora_create(C.byref(P))
        if not self._h:
            raise RuntimeError("oracle setup failed")

    @property
    def fine_lambda(self) -> float:
        return lib().ora_fine_lambda(self._h)

    def step(self) -> Report:
        r = Report()
        st = lib().ora_step(self._h, C.byref(r))
        if st != 0:
            raise RuntimeError(f"oracle step failed with status {st} at it={r.it}")
        return r

    def fields(self):
        u = [np.zeros(self.nv) for _ in range(3)]
        p = np.zeros(self.nc)
        lib().ora_get(self._h, *[_ptr(x) for x in u], _ptr(p))
        return u[0], u[1], u[2], p

    def set_fields(self, u0, u1, u2, p):
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (u0, u1, u2, p)]
        lib().ora_set(self._h, *[_ptr(x) for x in arrs])

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ora_destroy(self._h)
            self._h = None
