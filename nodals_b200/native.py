"""ctypes binding of the C ABI in include/nodals_b200.h.

The library is built in-tree (``python -m nodals_b200.build``) and loaded
from ``nodals_b200/_lib``.  There is no fallback: if the library is missing
the import fails with the build command to run.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libnodals_b200.so"
_lib = None

NDS_OK = 0
ERRORS = {-1: "NDS_E_INVALID", -2: "NDS_E_SETUP", -3: "NDS_E_CUDA", -4: "NDS_E_BREAKDOWN",
          -5: "NDS_E_NOT_CONVERGED", -6: "NDS_E_STATE"}

PRECISION = {"fp64": 0, "fp32": 1, "amg_fp32": 2, "mixed": 3}
KRYLOV = {"pcg": 0, "fgmres": 1}
RUN_MODE = {"fixed10": 0, "converge": 1}
MOMENTUM_WORK = {"fgs1": 0, "altgs1": 1, "sgs1": 2}
PRESSURE_SOLVER = {"pcg": 0, "richardson": 1, "cheb": 2}
AMG_HIERARCHY = {"sa": 0, "cf": 1}
AMG_SMOOTHER = {"cheb2": 0, "jacobi": 1, "l1jacobi": 2, "mcgs": 3}
SPECTRUM = {"auto": 0, "always": 1, "off": 2}
MCGS_ORDER = {"symmetric": 0, "forward": 1, "backward": 2}
CF_INTERP = {"direct": 0, "exti": 1}
_ENUMS = {"precision": PRECISION, "run_mode": RUN_MODE, "momentum_work": MOMENTUM_WORK,
          "pressure_solver": PRESSURE_SOLVER, "amg_hierarchy": AMG_HIERARCHY, "amg_smoother": AMG_SMOOTHER,
          "amg_spectrum_policy": SPECTRUM, "amg_mcgs_order": MCGS_ORDER, "cf_interp": CF_INTERP,
          "p_krylov": KRYLOV}


class NdsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [
        ("re", C.c_double), ("bulk", C.c_double), ("simple_tol", C.c_double), ("alpha_u", C.c_double),
        ("alpha_p", C.c_double), ("rau_scale", C.c_double),
        ("max_outer", C.c_int), ("run_mode", C.c_int), ("momentum_work", C.c_int),
        ("mom_omega", C.c_double), ("mom_rtol", C.c_double), ("mom_atol", C.c_double), ("mom_drop", C.c_double),
        ("mom_max", C.c_int),
        ("pressure_solver", C.c_int),
        ("p_rtol", C.c_double), ("p_atol", C.c_double),
        ("p_max", C.c_int),
        ("snapshot_tol", C.c_double),
        ("fine_csr_refresh_every", C.c_int),
        ("p_richardson_omega", C.c_double),
        ("p_cheb_degree", C.c_int), ("p_power_its", C.c_int),
        ("p_cheb_low_fraction", C.c_double), ("p_power_safety", C.c_double),
        ("amg_hierarchy", C.c_int), ("amg_smoother", C.c_int), ("amg_terminal", C.c_int),
        ("amg_spectrum_policy", C.c_int),
        ("amg_power_its", C.c_int), ("amg_cheb_degree", C.c_int),
        ("amg_lambda_safety", C.c_double), ("amg_lambda_low_fraction", C.c_double), ("amg_jacobi_omega", C.c_double),
        ("amg_jacobi_fine_sweeps", C.c_int), ("amg_jacobi_coarse_sweeps", C.c_int),
        ("amg_mcgs_omega", C.c_double),
        ("amg_mcgs_fine_sweeps", C.c_int), ("amg_mcgs_coarse_sweeps", C.c_int), ("amg_mcgs_order", C.c_int),
        ("cf_theta", C.c_double),
        ("cf_pmax", C.c_int), ("cf_interp", C.c_int), ("cf_aggressive_first", C.c_int),
        ("wall", C.c_char * 64), ("inlet", C.c_char * 64), ("outlet", C.c_char * 64),
        ("precision", C.c_int), ("threads", C.c_int), ("device", C.c_int), ("verbose", C.c_int),
        ("supg", C.c_int), ("supg_tau_scale", C.c_double), ("supg_magic", C.c_double),
        ("p_krylov", C.c_int), ("p_restart", C.c_int), ("p_inner_rtol", C.c_double), ("p_refine_max", C.c_int),
        ("p_guess", C.c_int), ("learned", C.c_int), ("geom_from_inlet", C.c_int), ("p_guess_fresh", C.c_int),
        ("amg_half", C.c_int),
    ]

    @classmethod
    def make(cls, **kw) -> "Options":
        o = cls()
        lib().nds_options_default(C.byref(o))
        for k, v in kw.items():
            if k in _ENUMS and isinstance(v, str):
                v = _ENUMS[k][v]
            if k in ("wall", "inlet", "outlet"):
                v = v.encode()
            if not hasattr(o, k):
                raise KeyError(f"unknown option {k}")
            setattr(o, k, v)
        return o


class IterReport(C.Structure):
    _fields_ = [("it", C.c_int), ("rel_cont", C.c_double), ("cont_norm", C.c_double), ("p_its", C.c_int),
                ("p_rel", C.c_double), ("audited", C.c_int), ("audit_rel", C.c_double * 3),
                ("all_momentum_met", C.c_int), ("converged", C.c_int),
                ("ms_assembly", C.c_double), ("ms_momentum", C.c_double), ("ms_continuity", C.c_double),
                ("ms_pressure", C.c_double), ("ms_update", C.c_double), ("ms_refresh", C.c_double)]


class SolveReport(C.Structure):
    _fields_ = [("outer_its", C.c_int), ("converged", C.c_int), ("pressure_all", C.c_int), ("finite_all", C.c_int),
                ("final_rel_cont", C.c_double), ("final_audit_rel", C.c_double * 3),
                ("avg_pressure_its", C.c_double), ("loop_ms", C.c_double), ("assembly_ms", C.c_double),
                ("momentum_ms", C.c_double), ("continuity_ms", C.c_double), ("pressure_ms", C.c_double),
                ("update_ms", C.c_double)]


class HpErrors(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("h_eff", "u_l2", "u_rel_l2", "p_shifted_l2", "p_shifted_rel_l2",
                                          "pressure_shift", "dp_fit", "dp_exact", "dp_rel_err")]


class ProfileEntry(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("calls", C.c_longlong), ("total_ms", C.c_double)]


class _Array(C.Structure):
    _fields_ = [("data", C.c_void_p), ("count", C.c_int64), ("dtype", C.c_int)]


_DT = {0: np.float64, 1: np.int32, 2: np.int64, 3: np.uint8, 4: np.uint32}


class HybridFlowOptions(C.Structure):
    """nds_hybrid_flow_options: the mixed-mesh pipe SIMPLE and its pressure
    preconditioner (defaults: the reference HXT4B binary, AMG fields those of
    its turbulent entry)."""
    _fields_ = ([(n, C.c_double) for n in ("re", "bulk", "gamma", "alpha_u", "alpha_p", "rau_scale", "simple_tol")]
                + [("max_outer", C.c_int), ("momentum_work", C.c_int)]
                + [(n, C.c_double) for n in ("mom_omega", "mom_rtol", "mom_atol", "p_rtol", "p_atol")]
                + [("p_max", C.c_int)]
                + [(n, C.c_int) for n in ("pressure_solver", "amg_smoother", "amg_spectrum_policy", "amg_terminal",
                                          "amg_power_its", "amg_cheb_degree", "amg_jacobi_fine_sweeps",
                                          "amg_jacobi_coarse_sweeps", "amg_mcgs_fine_sweeps", "amg_mcgs_coarse_sweeps",
                                          "amg_mcgs_order", "cf_pmax", "cf_interp", "cf_aggressive_first")]
                + [(n, C.c_double) for n in ("cf_theta", "amg_lambda_safety", "amg_lambda_low_fraction",
                                             "amg_jacobi_omega", "amg_mcgs_omega")]
                + [("amg_separate_post", C.c_int)])

    @classmethod
    def make(cls, **kw) -> "HybridFlowOptions":
        o = cls()
        lib().nds_hybrid_flow_defaults(C.byref(o))
        for k, v in kw.items():
            if not hasattr(o, k):
                raise AttributeError(f"no hybrid flow option {k}")
            setattr(o, k, v)
        return o


class HybridFlowReport(C.Structure):
    _fields_ = ([(n, C.c_int) for n in ("outer_its", "converged", "pass_", "n_hex", "n_tet", "n_velocity")]
                + [(n, C.c_double) for n in ("final_rel_cont", "avg_pressure_cg", "slope", "slope_exact", "p_in",
                                             "p_out", "drop", "drop_exact", "profile_rel_l2", "transverse_rel_l2",
                                             "conv_norm", "velocity_norm", "loop_ms")])


def _array_copy(a) -> np.ndarray:
    dt = np.dtype(_DT[a.dtype])
    if a.count == 0:
        return np.zeros(0, dtype=dt)
    buf = (C.c_char * (a.count * dt.itemsize)).from_address(a.data)
    return np.frombuffer(buf, dtype=dt).copy()


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise ImportError(f"{_LIB_PATH} is missing; build it with `python -m nodals_b200.build`")
        L = C.CDLL(str(_LIB_PATH))
        vp = C.c_void_p
        L.nds_last_error.restype = C.c_char_p
        L.nds_version.restype = C.c_char_p
        L.nds_options_default.argtypes = [C.POINTER(Options)]
        L.nds_mesh_read_polymesh.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.nds_mesh_read_msh2.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.nds_mesh_read_hxt1.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.nds_mesh_from_arrays.argtypes = [C.c_int, vp, C.c_int, vp, C.c_int, vp, vp, C.c_int, C.POINTER(C.c_char_p),
                                           C.POINTER(vp)]
        L.nds_mesh_counts.argtypes = [vp] + [C.POINTER(C.c_int)] * 4
        L.nds_mesh_destroy.argtypes = [vp]
        L.nds_problem_create.argtypes = [vp, C.POINTER(Options), C.POINTER(vp)]
        L.nds_problem_array.argtypes = [vp, C.c_char_p, C.POINTER(_Array)]
        L.nds_problem_counts.argtypes = [vp] + [C.POINTER(C.c_int)] * 4
        L.nds_problem_destroy.argtypes = [vp]
        L.nds_write_vtu.argtypes = [vp, C.c_char_p, vp, vp, vp, vp, C.c_int, C.c_int]
        L.nds_compute_hp_errors.argtypes = [vp, vp, vp, vp, vp, C.POINTER(HpErrors)]
        L.nds_cell_average_velocity.argtypes = [vp, vp, vp, vp, vp]
        L.nds_hybrid_flow_defaults.argtypes = [C.POINTER(HybridFlowOptions)]
        L.nds_hybrid_counts.argtypes = [C.c_char_p, C.POINTER(C.c_uint64)]
        L.nds_hybrid_write_vtu.argtypes = [C.c_char_p, C.c_char_p, vp, vp, vp, vp]
        L.nds_hybrid_amg_create.argtypes = [C.c_char_p, vp, C.POINTER(HybridFlowOptions), C.POINTER(vp)]
        L.nds_hybrid_amg_array.argtypes = [vp, C.c_char_p, C.POINTER(_Array)]
        L.nds_hybrid_amg_destroy.argtypes = [vp]
        L.nds_hybrid_flow_setup.argtypes = [C.c_char_p, C.POINTER(HybridFlowOptions), C.POINTER(vp)]
        if hasattr(L, "nds_hybrid_amg_vcycle"):
            L.nds_hybrid_amg_vcycle.argtypes = [C.c_char_p, vp, C.POINTER(HybridFlowOptions), C.c_int, vp, vp]
        if hasattr(L, "nds_hybrid_flow_fields"):
            L.nds_hybrid_flow_fields.argtypes = [C.c_char_p, C.POINTER(HybridFlowOptions), C.c_int, C.c_int,
                                                 C.POINTER(HybridFlowReport), vp, vp, vp, vp]
        if hasattr(L, "nds_solver_create"):
            L.nds_solver_create.argtypes = [vp, C.POINTER(vp)]
            L.nds_solver_reset.argtypes = [vp]
            L.nds_simple_step.argtypes = [vp, C.POINTER(IterReport)]
            L.nds_solve.argtypes = [vp, C.POINTER(SolveReport)]
            L.nds_get_fields.argtypes = [vp] * 5
            L.nds_set_fields.argtypes = [vp] * 5
            L.nds_simple_step_io.argtypes = [vp] * 9 + [C.POINTER(IterReport)]
            L.nds_solver_destroy.argtypes = [vp]
            L.nds_profile_enable.argtypes = [vp, C.c_int]
            L.nds_launch_count.restype = C.c_ulonglong
            L.nds_profile_read.argtypes = [vp, C.POINTER(ProfileEntry), C.c_int, C.POINTER(C.c_int)]
        if hasattr(L, "nds_mpnn_create"):
            L.nds_mpnn_create.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
            L.nds_mpnn_set_params.argtypes = [vp, vp, C.c_int]
            L.nds_mpnn_get_params.argtypes = [vp, vp, C.c_int]
            L.nds_mpnn_get_grads.argtypes = [vp, vp, C.c_int]
            L.nds_mpnn_forward.argtypes = [vp, C.c_void_p, C.c_int, vp, vp, vp]
            L.nds_mpnn_loss_backward.argtypes = [vp, C.c_void_p, C.c_int, vp, vp, vp, C.POINTER(C.c_double)]
            L.nds_mpnn_adam_step.argtypes = [vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int]
            L.nds_mpnn_backward.argtypes = [vp, C.c_void_p, vp]
            L.nds_solver_apply_operator.argtypes = [vp, vp, vp]
            L.nds_mpnn_activations.argtypes = [vp, C.c_int, vp]
            L.nds_mpnn_destroy.argtypes = [vp]
            L.nds_solver_load_stage.argtypes = [vp, vp, C.c_int]
            L.nds_solver_stage_graph.argtypes = [vp, vp, vp, vp]
            L.nds_solver_pressure_pair.argtypes = [vp, vp, vp]
            L.nds_solver_stage_counts.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        _lib = L
    return _lib


def _check(rc: int):
    if rc != NDS_OK:
        raise NdsError(rc, lib().nds_last_error().decode(errors="replace"))


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Mesh:
    def __init__(self, handle):
        self._h = handle

    @classmethod
    def read_polymesh(cls, path) -> "Mesh":
        h = C.c_void_p()
        _check(lib().nds_mesh_read_polymesh(str(path).encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def read_msh2(cls, path) -> "Mesh":
        h = C.c_void_p()
        _check(lib().nds_mesh_read_msh2(str(path).encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def read_hxt1(cls, path) -> "Mesh":
        h = C.c_void_p()
        _check(lib().nds_mesh_read_hxt1(str(path).encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def from_tetmesh(cls, m) -> "Mesh":
        """From a nodals_b200.meshgen.TetMesh (points, tets, tagged boundary triangles)."""
        from .meshgen import PATCHES
        xyz = np.ascontiguousarray(m.points, dtype=np.float64)
        tets = np.ascontiguousarray(m.tets, dtype=np.int32)
        btri = np.ascontiguousarray(m.bfaces, dtype=np.int32)
        bpat = np.ascontiguousarray(m.btag, dtype=np.int32)
        names = (C.c_char_p * len(PATCHES))(*[p.encode() for p in PATCHES])
        h = C.c_void_p()
        _check(lib().nds_mesh_from_arrays(len(xyz), _p(xyz), len(tets), _p(tets), len(btri), _p(btri), _p(bpat),
                                          len(PATCHES), names, C.byref(h)))
        return cls(h)

    def counts(self):
        v = [C.c_int() for _ in range(4)]
        _check(lib().nds_mesh_counts(self._h, *[C.byref(x) for x in v]))
        return dict(zip(("points", "cells", "faces", "internal"), (x.value for x in v)))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.nds_mesh_destroy(self._h)
            self._h = None


def hybrid_counts(path) -> tuple:
    c = (C.c_uint64 * 13)()
    _check(lib().nds_hybrid_counts(str(path).encode(), c))
    return tuple(int(x) for x in c)


def hybrid_flow(path, options: HybridFlowOptions | None = None, device: int = 0, verbose: int = 0, **kw):
    """Mixed-mesh pipe SIMPLE on the GPU; returns (report, u0, u1, u2, p)."""
    o = options if options is not None else HybridFlowOptions.make(**kw)
    n = hybrid_counts(path)
    u = [np.zeros(n[5]) for _ in range(3)]
    p = np.zeros(n[6])
    r = HybridFlowReport()
    _check(lib().nds_hybrid_flow_fields(str(path).encode(), C.byref(o), device, verbose, C.byref(r),
                                        *[_p(x) for x in (*u, p)]))
    return r, u[0], u[1], u[2], p


def hybrid_amg_vcycle(path, rau: np.ndarray, b: np.ndarray, options: HybridFlowOptions | None = None, device: int = 0,
                      **kw) -> np.ndarray:
    """z = M^-1 b for the mixed-mesh pressure AMG built and refreshed from rau (GPU)."""
    o = options if options is not None else HybridFlowOptions.make(**kw)
    r = np.ascontiguousarray(rau, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    z = np.zeros_like(bb)
    _check(lib().nds_hybrid_amg_vcycle(str(path).encode(), _p(r), C.byref(o), device, _p(bb), _p(z)))
    return z


class HybridAmg:
    """Host setup of the mixed-mesh pressure preconditioner for a given rAU
    (``rau`` given) or of the whole pipe SIMPLE (``rau`` None)."""

    def __init__(self, path, rau: np.ndarray | None, options: HybridFlowOptions | None = None, **kw):
        o = options if options is not None else HybridFlowOptions.make(**kw)
        h = C.c_void_p()
        if rau is None:
            _check(lib().nds_hybrid_flow_setup(str(path).encode(), C.byref(o), C.byref(h)))
        else:
            r = np.ascontiguousarray(rau, dtype=np.float64)
            _check(lib().nds_hybrid_amg_create(str(path).encode(), _p(r), C.byref(o), C.byref(h)))
        self._h = h

    def array(self, name: str) -> np.ndarray:
        a = _Array()
        _check(lib().nds_hybrid_amg_array(self._h, name.encode(), C.byref(a)))
        return _array_copy(a)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.nds_hybrid_amg_destroy(self._h)
            self._h = None


class Problem:
    """Host setup: numbering, momentum CSR, colouring, cell plans, AMG hierarchy."""

    def __init__(self, mesh: Mesh, options: Options | None = None, **kw):
        self.mesh = mesh
        self.options = options if options is not None else Options.make(**kw)
        h = C.c_void_p()
        _check(lib().nds_problem_create(mesh._h, C.byref(self.options), C.byref(h)))
        self._h = h

    def array(self, name: str) -> np.ndarray:
        a = _Array()
        _check(lib().nds_problem_array(self._h, name.encode(), C.byref(a)))
        dt = np.dtype(_DT[a.dtype])
        if a.count == 0:
            return np.zeros(0, dtype=dt)
        buf = (C.c_char * (a.count * dt.itemsize)).from_address(a.data)
        return np.frombuffer(buf, dtype=dt).copy()

    def scalar(self, name: str) -> float:
        return float(self.array(name)[0])

    def counts(self):
        v = [C.c_int() for _ in range(4)]
        _check(lib().nds_problem_counts(self._h, *[C.byref(x) for x in v]))
        return dict(zip(("nc", "nv", "ncolors", "levels"), (x.value for x in v)))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.nds_problem_destroy(self._h)
            self._h = None


class Solver:
    """Device solver over a Problem (the problem must outlive the solver)."""

    def __init__(self, problem: Problem):
        self.problem = problem
        h = C.c_void_p()
        _check(lib().nds_solver_create(problem._h, C.byref(h)))
        self._h = h
        c = problem.counts()
        self.nc, self.nv = c["nc"], c["nv"]

    def reset(self):
        _check(lib().nds_solver_reset(self._h))

    def step(self) -> IterReport:
        r = IterReport()
        _check(lib().nds_simple_step(self._h, C.byref(r)))
        return r

    def solve(self) -> SolveReport:
        r = SolveReport()
        _check(lib().nds_solve(self._h, C.byref(r)))
        return r

    def fields(self):
        u = [np.zeros(self.nv) for _ in range(3)]
        p = np.zeros(self.nc)
        _check(lib().nds_get_fields(self._h, *[_p(x) for x in u], _p(p)))
        return u[0], u[1], u[2], p

    def set_fields(self, u0, u1, u2, p):
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (u0, u1, u2, p)]
        _check(lib().nds_set_fields(self._h, *[_p(x) for x in arrs]))

    def step_io(self, inputs, outputs) -> IterReport:
        """One SIMPLE iteration with the state passed through host memory:
        inputs and outputs are (u0, u1, u2, p) sequences of float64 arrays
        (or None entries, or raw addresses of page-locked buffers as ints)."""
        def ptr(x):
            if x is None:
                return None
            if isinstance(x, int):
                return C.c_void_p(x)
            if x.dtype != np.float64 or not x.flags.c_contiguous:
                raise ValueError("step_io arrays must be contiguous float64")
            return _p(x)
        r = IterReport()
        _check(lib().nds_simple_step_io(self._h, *[ptr(x) for x in inputs], *[ptr(x) for x in outputs], C.byref(r)))
        return r

    def profile(self, enable: bool = True):
        _check(lib().nds_profile_enable(self._h, int(enable)))

    def profile_read(self) -> dict:
        buf = (ProfileEntry * 32)()
        n = C.c_int()
        _check(lib().nds_profile_read(self._h, buf, 32, C.byref(n)))
        return {buf[i].name.decode(): (buf[i].calls, buf[i].total_ms) for i in range(n.value)}

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.nds_solver_destroy(self._h)
            self._h = None


def launch_count() -> int:
    return int(lib().nds_launch_count())


def _f64(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def cell_average_velocity(problem: Problem, u0, u1, u2, out: np.ndarray | None = None) -> np.ndarray:
    """U0 cell averages (1/4 vertex + 9/40 face bubbles), shape (nc, 3)."""
    a = [_f64(x) for x in (u0, u1, u2)]
    res = np.zeros((problem.counts()["nc"], 3))
    _check(lib().nds_cell_average_velocity(problem._h, *[_p(x) for x in a], _p(res)))
    if out is not None:
        out[...] = res
    return res


def hp_errors(problem: Problem, u0, u1, u2, p) -> dict:
    a = [_f64(x) for x in (u0, u1, u2, p)]
    e = HpErrors()
    _check(lib().nds_compute_hp_errors(problem._h, *[_p(x) for x in a], C.byref(e)))
    return {k: getattr(e, k) for k, _ in HpErrors._fields_}


def write_vtu(problem: Problem, path, u0, u1, u2, p, converged: bool = False, outer_its: int = 0):
    a = [_f64(x) for x in (u0, u1, u2, p)]
    _check(lib().nds_write_vtu(problem._h, str(path).encode(), *[_p(x) for x in a], int(converged), int(outer_its)))


# ---------------------------------------------------------------- learned stage
class MpnnGraph(C.Structure):
    _fields_ = [("n", C.c_int), ("nbr", C.c_void_p), ("ew", C.c_void_p), ("dscale", C.c_void_p)]


MPNN_NPARAM = 25026


class Mpnn:
    """Device state of the learned stage's network (nds_mpnn_*): graphs of up
    to n_max nodes; training=True keeps activations, gradients, Adam moments.
    Arrays passed in are device addresses (ints) or objects with data_ptr()."""

    def __init__(self, n_max: int, training: bool = False, device: int = 0):
        h = C.c_void_p()
        _check(lib().nds_mpnn_create(int(n_max), int(training), int(device), C.byref(h)))
        self._h = h

    @staticmethod
    def _addr(x):
        if x is None:
            return None
        return C.c_void_p(x if isinstance(x, int) else x.data_ptr())

    def graph(self, n, nbr, ew, dscale) -> MpnnGraph:
        """The graph view over device arrays; it holds raw addresses, so the
        caller keeps nbr, ew and dscale alive while the view is used."""
        return MpnnGraph(int(n), self._addr(nbr), self._addr(ew), self._addr(dscale))

    def set_params(self, p: np.ndarray):
        a = np.ascontiguousarray(p, dtype=np.float32)
        _check(lib().nds_mpnn_set_params(self._h, a.ctypes.data_as(C.c_void_p), MPNN_NPARAM))

    def params(self) -> np.ndarray:
        a = np.zeros(MPNN_NPARAM, dtype=np.float32)
        _check(lib().nds_mpnn_get_params(self._h, a.ctypes.data_as(C.c_void_p), MPNN_NPARAM))
        return a

    def grads(self) -> np.ndarray:
        a = np.zeros(MPNN_NPARAM, dtype=np.float32)
        _check(lib().nds_mpnn_get_grads(self._h, a.ctypes.data_as(C.c_void_p), MPNN_NPARAM))
        return a

    @staticmethod
    def _segs(segs):
        if segs is None:
            return 0, None
        s = np.ascontiguousarray(segs, dtype=np.int32)
        return len(s) - 1, s

    def forward(self, g: MpnnGraph, v, z, segs=None):
        ns, s = self._segs(segs)
        _check(lib().nds_mpnn_forward(self._h, C.byref(g), ns, None if s is None else s.ctypes.data_as(C.c_void_p),
                                      self._addr(v), self._addr(z)))

    def loss_backward(self, g: MpnnGraph, v, x, segs=None) -> float:
        ns, s = self._segs(segs)
        loss = C.c_double()
        _check(lib().nds_mpnn_loss_backward(self._h, C.byref(g), ns,
                                            None if s is None else s.ctypes.data_as(C.c_void_p), self._addr(v),
                                            self._addr(x), C.byref(loss)))
        return loss.value

    def backward(self, g: MpnnGraph, dz):
        """Gradients from dL/dz of the last forward on the same graph."""
        _check(lib().nds_mpnn_backward(self._h, C.byref(g), self._addr(dz)))

    def adam_step(self, lr: float, step: int, beta1=0.9, beta2=0.999, eps=1e-8):
        _check(lib().nds_mpnn_adam_step(self._h, C.c_float(lr), C.c_float(beta1), C.c_float(beta2), C.c_float(eps),
                                        int(step)))

    def activations(self, layer: int, out):
        _check(lib().nds_mpnn_activations(self._h, int(layer), self._addr(out)))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.nds_mpnn_destroy(self._h)
            self._h = None


def solver_load_stage(solver: "Solver", params: np.ndarray):
    a = np.ascontiguousarray(params, dtype=np.float32)
    _check(lib().nds_solver_load_stage(solver._h, a.ctypes.data_as(C.c_void_p), MPNN_NPARAM))


def solver_stage_graph(solver: "Solver", nbr, ew, dscale):
    _check(lib().nds_solver_stage_graph(solver._h, Mpnn._addr(nbr), Mpnn._addr(ew), Mpnn._addr(dscale)))


def solver_pressure_pair(solver: "Solver", rhs, x):
    _check(lib().nds_solver_pressure_pair(solver._h, Mpnn._addr(rhs), Mpnn._addr(x)))


def solver_apply_operator(solver: "Solver", x, y):
    """y = A x with the solver's current FP32 pressure operator (device arrays)."""
    _check(lib().nds_solver_apply_operator(solver._h, Mpnn._addr(x), Mpnn._addr(y)))


def solver_stage_counts(solver: "Solver"):
    a, f = C.c_longlong(), C.c_longlong()
    _check(lib().nds_solver_stage_counts(solver._h, C.byref(a), C.byref(f)))
    return a.value, f.value
