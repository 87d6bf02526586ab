"""``.case`` front end: translate an annotated case file into the H8 command line
and launch the drop-in executable.

Behaviour of the reference launcher (scripts/nodals_gpu_case.py:23-328):
strict INI sections/keys, ``--set SECTION.KEY=VALUE`` overrides, case defaults
that differ from the binary defaults (cf / jacobi / richardson / fp32 /
converge / simple rtol 1e-3), ``--dry-run``, ``--dump-options-json``,
``--exe``, the NODALS_GPU_{FP32,FP64}_EXE environment overrides, a tee'd log,
and the runner exit codes 0 pass, 2 missing solver, 4 configuration error,
21 not converged, 124 timeout.  Usage::

    python -m nodals_b200.case my.case [--dry-run] [--set pressure.rtol=1e-4] [-- extra flags]
"""
from __future__ import annotations

import argparse
import configparser
import datetime as _dt
import json
import os
import shlex
import subprocess
import sys
from pathlib import Path
from typing import Dict, Iterable, List

_TRUE = {"1", "true", "yes", "on"}
_FALSE = {"0", "false", "no", "off"}

# section -> accepted keys (the reference's case schema)
SCHEMA: Dict[str, frozenset] = {
    "run": frozenset({"name", "precision", "run_mode", "output_root", "timeout_seconds"}),
    "solver": frozenset({"mesh", "re", "bulk_velocity"}),
    "boundary": frozenset({"wall_patch", "inlet_patch", "outlet_patch"}),
    "simple": frozenset({"rtol", "max_iterations", "alpha_u", "alpha_p"}),
    "momentum": frozenset({"work", "rtol", "atol", "relative_drop", "omega", "max_iterations"}),
    "supg": frozenset({"enabled", "tau_scale", "magic", "form", "quad_points"}),
    "pressure": frozenset({"solver", "rtol", "atol", "max_iterations", "snapshot_tolerance", "fine_csr_refresh_every",
                           "richardson_omega", "chebyshev_degree", "power_iterations", "chebyshev_low_fraction",
                           "power_safety"}),
    "pressure_amg": frozenset({"hierarchy", "smoother", "terminal_rows", "spectrum_policy", "power_iterations",
                               "chebyshev_degree", "lambda_safety", "lambda_low_fraction", "jacobi_omega"}),
    "pressure_amg_cf": frozenset({"coarsening", "strength", "theta", "interpolation", "pmax", "aggressive_first"}),
}
KNOWN_KEYS = SCHEMA  # name used by the reference module

PACKAGE_LIB = Path(__file__).resolve().parent / "_lib"
DEFAULT_CASE = Path(__file__).resolve().parent / "cases" / "gpu-h8-annotated.case"


def _expand(v: str) -> str:
    return os.path.expandvars(os.path.expanduser(v.strip()))


def _as_bool(v: str, where: str) -> bool:
    s = str(v).strip().lower()
    if s in _TRUE:
        return True
    if s in _FALSE:
        return False
    raise ValueError(f"{where}: expected boolean, got {v!r}")


def _validate_case_keys(cp: configparser.ConfigParser) -> None:
    for sec in cp.sections():
        if sec not in SCHEMA:
            raise ValueError(f"unknown GPU case section [{sec}]")
        for key, _ in cp.items(sec):
            if key not in SCHEMA[sec]:
                raise ValueError(f"unknown GPU case key [{sec}] {key}")


def _read_case(path: Path) -> configparser.ConfigParser:
    cp = configparser.ConfigParser(interpolation=None, inline_comment_prefixes=("#", ";"))
    cp.optionxform = str.lower
    with Path(path).open("r", encoding="utf-8") as f:
        cp.read_file(f)
    _validate_case_keys(cp)
    return cp


read_case = _read_case


def _get(cp, sec, key, default=None):
    if cp.has_option(sec, key):
        return cp.get(sec, key).strip()
    return default


def _require(cp, sec, key) -> str:
    v = _get(cp, sec, key)
    if v is None or v == "":
        raise ValueError(f"missing required [{sec}] {key}")
    return v


def _case_overrides(cp: configparser.ConfigParser, overrides: Iterable[str]) -> None:
    for item in overrides:
        if "=" not in item or "." not in item.split("=", 1)[0]:
            raise ValueError(f"--set expects section.key=value, got {item!r}")
        lhs, value = item.split("=", 1)
        sec, key = (x.strip().lower() for x in lhs.split(".", 1))
        if sec not in SCHEMA:
            raise ValueError(f"unknown GPU case section [{sec}]")
        if key not in SCHEMA[sec]:
            raise ValueError(f"unknown GPU case key [{sec}] {key}")
        if not cp.has_section(sec):
            cp.add_section(sec)
        cp.set(sec, key, value)


def build_gpu_options(cp: configparser.ConfigParser) -> List[str]:
    """Map a case onto the H8 argv, flag by flag (nodals_gpu_case.py:112-220)."""
    _validate_case_keys(cp)
    argv: List[str] = []

    def flag(name, value):
        argv.extend([f"--{name}", str(value)])

    name = _get(cp, "run", "name", "nodals_gpu")
    run_mode = str(_get(cp, "run", "run_mode", "converge")).lower()
    if run_mode not in ("fixed10", "converge"):
        raise ValueError("[run] run_mode must be fixed10 or converge")
    flag("mesh", _expand(_require(cp, "solver", "mesh")))
    flag("tag", name)
    flag("wall", _get(cp, "boundary", "wall_patch", "patch_0_0"))
    flag("inlet", _get(cp, "boundary", "inlet_patch", "patch_2_0"))
    flag("outlet", _get(cp, "boundary", "outlet_patch", "patch_1_0"))
    flag("re", _get(cp, "solver", "re", "20"))
    flag("bulk", _get(cp, "solver", "bulk_velocity", "1.0"))

    max_outer = int(str(_get(cp, "simple", "max_iterations", "2500")))
    if run_mode == "fixed10" and max_outer != 10:
        raise ValueError("[run] run_mode=fixed10 requires [simple] max_iterations=10")
    flag("simple-tol", _get(cp, "simple", "rtol", "1e-3"))
    flag("max-outer", max_outer)
    flag("alpha-u", _get(cp, "simple", "alpha_u", "0.5"))
    flag("alpha-p", _get(cp, "simple", "alpha_p", "0.5"))

    work = str(_get(cp, "momentum", "work", "fgs1")).lower()
    if work != "fgs1":
        raise ValueError("current H8 supports only [momentum] work=fgs1")
    flag("mom-rtol", _get(cp, "momentum", "rtol", "1e-6"))
    flag("mom-atol", _get(cp, "momentum", "atol", "1e-12"))
    flag("mom-drop", _get(cp, "momentum", "relative_drop", "0.1"))
    flag("mom-omega", _get(cp, "momentum", "omega", "1.0"))
    flag("mom-max", _get(cp, "momentum", "max_iterations", "20000"))

    supg = _as_bool(str(_get(cp, "supg", "enabled", "false")), "[supg] enabled")
    supg_form = str(_get(cp, "supg", "form", "implicit")).lower()
    supg_quad = int(str(_get(cp, "supg", "quad_points", "64")))
    if supg and supg_form != "implicit":
        raise ValueError("current H8 GPU SUPG supports only [supg] form=implicit")
    if supg and supg_quad != 64:
        raise ValueError("current H8 GPU SUPG supports only [supg] quad_points=64")
    flag("supg", 1 if supg else 0)
    flag("supg-tau-scale", _get(cp, "supg", "tau_scale", "0.05"))
    flag("supg-magic", _get(cp, "supg", "magic", "9.0"))
    flag("supg-form", supg_form)
    flag("supg-quad-points", supg_quad)

    psolver = str(_get(cp, "pressure", "solver", "richardson")).lower()
    if psolver not in ("pcg", "richardson", "cheb"):
        raise ValueError("[pressure] solver must be pcg, richardson, or cheb")
    flag("p-rtol", _get(cp, "pressure", "rtol", "0.5"))
    flag("p-atol", _get(cp, "pressure", "atol", "1e-12"))
    flag("p-max", _get(cp, "pressure", "max_iterations", "20"))
    flag("snapshot-tol", _get(cp, "pressure", "snapshot_tolerance", "5e-6"))
    refresh = int(str(_get(cp, "pressure", "fine_csr_refresh_every", "1")))
    if refresh != 1:
        raise ValueError("current H8 requires [pressure] fine_csr_refresh_every=1")
    flag("fine-csr-refresh-every", refresh)
    flag("pressure-solver", psolver)
    flag("pressure-richardson-omega", _get(cp, "pressure", "richardson_omega", "1.0"))
    flag("pressure-cheb-degree", _get(cp, "pressure", "chebyshev_degree", "3"))
    flag("pressure-power-its", _get(cp, "pressure", "power_iterations", "6"))
    flag("pressure-cheb-low-fraction", _get(cp, "pressure", "chebyshev_low_fraction", "0.05"))
    flag("pressure-power-safety", _get(cp, "pressure", "power_safety", "1.15"))

    hierarchy = str(_get(cp, "pressure_amg", "hierarchy", "cf")).lower()
    if hierarchy not in ("sa", "cf"):
        raise ValueError("[pressure_amg] hierarchy must be sa or cf")
    smoother = str(_get(cp, "pressure_amg", "smoother", "jacobi")).lower()
    if smoother not in ("cheb2", "jacobi", "l1jacobi"):
        raise ValueError("[pressure_amg] smoother must be cheb2, jacobi, or l1jacobi")
    spectrum = str(_get(cp, "pressure_amg", "spectrum_policy", "auto")).lower()
    if spectrum not in ("auto", "always", "off"):
        raise ValueError("[pressure_amg] spectrum_policy must be auto, always, or off")
    if smoother == "cheb2" and spectrum == "off":
        raise ValueError("[pressure_amg] smoother=cheb2 requires spectrum_policy=auto or always")
    flag("amg-hierarchy", hierarchy)
    flag("amg-smoother", smoother)
    flag("amg-terminal", _get(cp, "pressure_amg", "terminal_rows", "1000"))
    flag("amg-spectrum-policy", spectrum)
    flag("amg-power-its", _get(cp, "pressure_amg", "power_iterations", "16"))
    flag("amg-cheb-degree", _get(cp, "pressure_amg", "chebyshev_degree", "2"))
    flag("amg-lambda-safety", _get(cp, "pressure_amg", "lambda_safety", "1.5"))
    flag("amg-lambda-low-fraction", _get(cp, "pressure_amg", "lambda_low_fraction", "0.05"))
    flag("amg-jacobi-omega", _get(cp, "pressure_amg", "jacobi_omega", "0.7"))

    coarsening = str(_get(cp, "pressure_amg_cf", "coarsening", "pmis")).lower()
    strength = str(_get(cp, "pressure_amg_cf", "strength", "classical-negative")).lower()
    interp = str(_get(cp, "pressure_amg_cf", "interpolation", "exti")).lower()
    if coarsening != "pmis":
        raise ValueError("current H8 CF hierarchy supports only [pressure_amg_cf] coarsening=pmis")
    if strength != "classical-negative":
        raise ValueError("current H8 CF hierarchy supports only [pressure_amg_cf] strength=classical-negative")
    if interp not in ("direct", "exti"):
        raise ValueError("[pressure_amg_cf] interpolation must be direct or exti")
    aggressive = _as_bool(str(_get(cp, "pressure_amg_cf", "aggressive_first", "false")), "[pressure_amg_cf] aggressive_first")
    flag("cf-coarsening", coarsening)
    flag("cf-strength", strength)
    flag("cf-theta", _get(cp, "pressure_amg_cf", "theta", "0.25"))
    flag("cf-interp", interp)
    flag("cf-pmax", _get(cp, "pressure_amg_cf", "pmax", "8"))
    flag("cf-aggressive-first", 1 if aggressive else 0)

    flag("momentum-work", work)
    flag("run-mode", run_mode)
    return argv


def _precision(cp: configparser.ConfigParser) -> str:
    p = str(_get(cp, "run", "precision", "fp32")).lower()
    if p not in ("fp32", "fp64"):
        raise ValueError("[run] precision must be fp32 or fp64")
    return p


def _find_solver(precision: str, explicit: str | None) -> Path:
    binary = f"nodals_gpu_h8_{precision}"
    cands: List[Path] = []
    if explicit:
        cands.append(Path(_expand(explicit)))
    env = os.environ.get(f"NODALS_GPU_{precision.upper()}_EXE")
    if env:
        cands.append(Path(_expand(env)))
    cands.append(PACKAGE_LIB / binary)
    for c in cands:
        if c.is_file() and os.access(c, os.X_OK):
            return c
    return cands[0]


def _tee(cmd: List[str], log: Path, timeout: int) -> int:
    log.parent.mkdir(parents=True, exist_ok=True)
    with log.open("w", encoding="utf-8", errors="replace") as f:
        proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, bufsize=1)
        try:
            assert proc.stdout is not None
            for line in proc.stdout:
                sys.stdout.write(line)
                sys.stdout.flush()
                f.write(line)
                f.flush()
            return proc.wait(timeout=None if timeout <= 0 else timeout)
        except subprocess.TimeoutExpired:
            proc.terminate()
            try:
                proc.wait(5)
            except subprocess.TimeoutExpired:
                proc.kill()
            return 124


def main(argv: List[str]) -> int:
    extra: List[str] = []
    if "--" in argv:
        i = argv.index("--")
        extra, argv = argv[i + 1:], argv[:i]
    ap = argparse.ArgumentParser(prog="nodals-gpu", description="Run the B200 SIMPLE solver from a .case file")
    ap.add_argument("case", type=Path)
    ap.add_argument("--dry-run", action="store_true")
    ap.add_argument("--dump-options-json", action="store_true")
    ap.add_argument("--exe", help="solver executable override")
    ap.add_argument("--set", action="append", default=[], metavar="SECTION.KEY=VALUE")
    ns = ap.parse_args(argv)
    case_path = ns.case.expanduser().resolve()
    cp = _read_case(case_path)
    _case_overrides(cp, ns.set)
    _validate_case_keys(cp)
    options = build_gpu_options(cp)
    precision = _precision(cp)
    solver = _find_solver(precision, ns.exe)
    name = str(_get(cp, "run", "name", case_path.stem))
    timeout = int(str(_get(cp, "run", "timeout_seconds", "0")))
    stamp = _dt.datetime.now().strftime("%Y%m%d_%H%M%S")
    out_cfg = str(_get(cp, "run", "output_root", "auto"))
    outroot = (Path.home() / "Downloads" / f"NodalS_GPU_{name}_{stamp}") if out_cfg.lower() == "auto" else Path(_expand(out_cfg))
    log = outroot / f"{name}.log"
    cmd = [str(solver)] + options + extra
    print(f"NODALS_GPU_CASE name={name} file={case_path} precision={precision} output={outroot}")
    print("NODALS_GPU_COMMAND " + shlex.join(cmd))
    if ns.dump_options_json:
        print("NODALS_GPU_OPTIONS_JSON=" + json.dumps(options))
    if ns.dry_run:
        print("NODALS_GPU_CASE_RESULT status=DRY_RUN")
        return 0
    if not solver.is_file() or not os.access(solver, os.X_OK):
        print(f"NODALS_GPU_CASE_RESULT status=FAIL reason=missing_solver executable={solver}", file=sys.stderr)
        return 2
    rc = _tee(cmd, log, timeout)
    print(f"NODALS_GPU_ARTIFACTS log={log} outroot={outroot}")
    if rc != 0:
        print(f"NODALS_GPU_CASE_RESULT status=FAIL rc={rc}")
        return rc
    text = log.read_text(encoding="utf-8", errors="replace")
    if any(l.startswith("NODALS_GPU_RESULT gate=H8 ") and "status=PASS" in l for l in text.splitlines()):
        print("NODALS_GPU_CASE_RESULT status=PASS")
        return 0
    print("NODALS_GPU_CASE_RESULT status=NOT_CONVERGED reason=no_NODALS_GPU_RESULT_PASS")
    return 21


def cli() -> int:
    try:
        return main(sys.argv[1:])
    except (ValueError, configparser.Error, OSError) as e:
        print(f"NODALS_GPU_CASE_ERROR {e}", file=sys.stderr)
        return 4


if __name__ == "__main__":
    raise SystemExit(cli())
