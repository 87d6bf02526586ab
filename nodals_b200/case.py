"""``.case`` front end: an annotated INI case file -> the drop-in H8 command line.

Interface kept from the reference launcher (``bin/nodals-gpu`` ->
``scripts/nodals_gpu_case.py``): the sections and keys of the case schema,
their defaults (which differ from the binary's own: CF/PMIS hierarchy, Jacobi
smoother, Richardson outer solver, fp32, converge mode, SIMPLE rtol 1e-3), the
error messages, ``--set SECTION.KEY=VALUE`` overrides, ``--dry-run``,
``--dump-options-json``, ``--exe`` and the ``NODALS_GPU_{FP32,FP64}_EXE``
variables, the ``NODALS_GPU_CASE*`` markers and the exit codes 0 pass,
2 missing solver, 4 configuration error, 21 not converged, 124 timeout.

Design: every key is one row of ``KEYS`` (section, key, CLI flag, default,
value rule).  The same table validates a case, fills defaults, and emits the
argv; the few cross-key rules are the functions in ``CROSS_RULES``.  Usage::

    python -m nodals_b200.case my.case [--dry-run] [--set pressure.rtol=1e-4] [-- extra flags]
"""
from __future__ import annotations

import argparse
import configparser
import datetime
import json
import os
import shlex
import subprocess
import sys
from dataclasses import dataclass
from pathlib import Path
from typing import Callable, Dict, List, Optional, Sequence, Tuple

PACKAGE_LIB = Path(__file__).resolve().parent / "_lib"
DEFAULT_CASE = Path(__file__).resolve().parent / "cases" / "gpu-h8-annotated.case"

EXIT_PASS, EXIT_NO_SOLVER, EXIT_CONFIG, EXIT_NOT_CONVERGED, EXIT_TIMEOUT = 0, 2, 4, 21, 124


def _or_list(words: Sequence[str]) -> str:
    """'a or b' / 'a, b, or c' (the wording of the schema's messages)."""
    if len(words) <= 2:
        return " or ".join(words)
    return ", ".join(words[:-1]) + ", or " + words[-1]


@dataclass(frozen=True)
class Key:
    """One case key.  ``flag``: the H8 option it becomes (None: read by the
    launcher only).  ``default``: None marks a required key.  ``kind``:
    'text' (passed through), 'path' (user and environment expansion),
    'lower' (lower-cased), 'int', 'bool' (true/false words -> 1/0).
    ``choices``: accepted values; ``only``: the single value the solver
    supports, with ``scope`` naming what imposes it."""
    section: str
    key: str
    flag: Optional[str]
    default: Optional[str]
    kind: str = "text"
    choices: Tuple[str, ...] = ()
    only: Optional[str] = None
    scope: str = "H8"


KEYS: Tuple[Key, ...] = (
    # [run]: launcher settings
    Key("run", "name", "tag", "nodals_gpu"),              # the log's name defaults to the case file's stem
    Key("run", "precision", None, "fp32", "lower", ("fp32", "fp64")),
    Key("run", "run_mode", "run-mode", "converge", "lower", ("fixed10", "converge")),
    Key("run", "output_root", None, "auto"),
    Key("run", "timeout_seconds", None, "0", "int"),
    # [solver], [boundary]: mesh and physics
    Key("solver", "mesh", "mesh", None, "path"),
    Key("solver", "re", "re", "20"),
    Key("solver", "bulk_velocity", "bulk", "1.0"),
    Key("boundary", "wall_patch", "wall", "patch_0_0"),
    Key("boundary", "inlet_patch", "inlet", "patch_2_0"),
    Key("boundary", "outlet_patch", "outlet", "patch_1_0"),
    # [simple]: outer loop
    Key("simple", "rtol", "simple-tol", "1e-3"),
    Key("simple", "max_iterations", "max-outer", "2500", "int"),
    Key("simple", "alpha_u", "alpha-u", "0.5"),
    Key("simple", "alpha_p", "alpha-p", "0.5"),
    # [momentum]
    Key("momentum", "work", "momentum-work", "fgs1", "lower", only="fgs1"),
    Key("momentum", "rtol", "mom-rtol", "1e-6"),
    Key("momentum", "atol", "mom-atol", "1e-12"),
    Key("momentum", "relative_drop", "mom-drop", "0.1"),
    Key("momentum", "omega", "mom-omega", "1.0"),
    Key("momentum", "max_iterations", "mom-max", "20000"),
    # [supg]: laminar streamline-upwind stabilisation
    Key("supg", "enabled", "supg", "false", "bool"),
    Key("supg", "tau_scale", "supg-tau-scale", "0.05"),
    Key("supg", "magic", "supg-magic", "9.0"),
    Key("supg", "form", "supg-form", "implicit", "lower"),
    Key("supg", "quad_points", "supg-quad-points", "64", "int"),
    # [pressure]: the outer pressure solver
    Key("pressure", "solver", "pressure-solver", "richardson", "lower", ("pcg", "richardson", "cheb")),
    Key("pressure", "rtol", "p-rtol", "0.5"),
    Key("pressure", "atol", "p-atol", "1e-12"),
    Key("pressure", "max_iterations", "p-max", "20"),
    Key("pressure", "snapshot_tolerance", "snapshot-tol", "5e-6"),
    Key("pressure", "fine_csr_refresh_every", "fine-csr-refresh-every", "1", "int"),
    Key("pressure", "richardson_omega", "pressure-richardson-omega", "1.0"),
    Key("pressure", "chebyshev_degree", "pressure-cheb-degree", "3"),
    Key("pressure", "power_iterations", "pressure-power-its", "6"),
    Key("pressure", "chebyshev_low_fraction", "pressure-cheb-low-fraction", "0.05"),
    Key("pressure", "power_safety", "pressure-power-safety", "1.15"),
    # [pressure_amg]: the V-cycle
    Key("pressure_amg", "hierarchy", "amg-hierarchy", "cf", "lower", ("sa", "cf")),
    Key("pressure_amg", "smoother", "amg-smoother", "jacobi", "lower", ("cheb2", "jacobi", "l1jacobi")),
    Key("pressure_amg", "terminal_rows", "amg-terminal", "1000"),
    Key("pressure_amg", "spectrum_policy", "amg-spectrum-policy", "auto", "lower", ("auto", "always", "off")),
    Key("pressure_amg", "power_iterations", "amg-power-its", "16"),
    Key("pressure_amg", "chebyshev_degree", "amg-cheb-degree", "2"),
    Key("pressure_amg", "lambda_safety", "amg-lambda-safety", "1.5"),
    Key("pressure_amg", "lambda_low_fraction", "amg-lambda-low-fraction", "0.05"),
    Key("pressure_amg", "jacobi_omega", "amg-jacobi-omega", "0.7"),
    # [pressure_amg_cf]: classical coarsening
    Key("pressure_amg_cf", "coarsening", "cf-coarsening", "pmis", "lower", only="pmis", scope="H8 CF hierarchy"),
    Key("pressure_amg_cf", "strength", "cf-strength", "classical-negative", "lower", only="classical-negative",
        scope="H8 CF hierarchy"),
    Key("pressure_amg_cf", "theta", "cf-theta", "0.25"),
    Key("pressure_amg_cf", "interpolation", "cf-interp", "exti", "lower", ("direct", "exti")),
    Key("pressure_amg_cf", "pmax", "cf-pmax", "8"),
    Key("pressure_amg_cf", "aggressive_first", "cf-aggressive-first", "false", "bool"),
)

SCHEMA: Dict[str, frozenset] = {}
for _k in KEYS:
    SCHEMA[_k.section] = SCHEMA.get(_k.section, frozenset()) | {_k.key}
_BY_NAME = {(k.section, k.key): k for k in KEYS}

_TRUE_WORDS, _FALSE_WORDS = ("1", "true", "yes", "on"), ("0", "false", "no", "off")


class Case:
    """A case file's values, checked against ``KEYS``."""

    def __init__(self, values: Dict[Tuple[str, str], str], path: Optional[Path] = None):
        self.values = values
        self.path = path
        self.check_names()

    @classmethod
    def read(cls, path) -> "Case":
        ini = configparser.ConfigParser(interpolation=None, inline_comment_prefixes=("#", ";"))
        ini.optionxform = str.lower
        with Path(path).open("r", encoding="utf-8") as f:
            ini.read_file(f)
        values = {(sec, key): val.strip() for sec in ini.sections() for key, val in ini.items(sec)}
        for sec in ini.sections():  # an empty unknown section is an error too
            if sec not in SCHEMA:
                raise ValueError(f"unknown GPU case section [{sec}]")
        return cls(values, Path(path))

    @staticmethod
    def check_name(sec: str, key: str) -> None:
        if sec not in SCHEMA:
            raise ValueError(f"unknown GPU case section [{sec}]")
        if key not in SCHEMA[sec]:
            raise ValueError(f"unknown GPU case key [{sec}] {key}")

    def check_names(self) -> None:
        for sec, key in self.values:
            self.check_name(sec, key)

    def set(self, section: str, key: str, value: str) -> None:
        self.check_name(section, key)
        self.values[(section, key)] = value

    def override(self, items: Sequence[str]) -> None:
        """Apply ``section.key=value`` items (``--set``)."""
        for item in items:
            lhs, eq, value = item.partition("=")
            sec, dot, key = lhs.partition(".")
            if not eq or not dot:
                raise ValueError(f"--set expects section.key=value, got {item!r}")
            self.set(sec.strip().lower(), key.strip().lower(), value)

    def raw(self, section: str, key: str) -> Optional[str]:
        v = self.values.get((section, key))
        return None if v is None else v.strip()

    def value(self, section: str, key: str):
        """The key's value after its default and rule (str, int or bool)."""
        spec = _BY_NAME[(section, key)]
        v = self.raw(section, key)
        if v is None:
            v = spec.default
        if v is None or v == "":
            raise ValueError(f"missing required [{section}] {key}")
        if spec.kind == "path":
            return os.path.expandvars(os.path.expanduser(v))
        if spec.kind == "int":
            return int(v)
        if spec.kind == "bool":
            w = v.lower()
            if w in _TRUE_WORDS:
                return True
            if w in _FALSE_WORDS:
                return False
            raise ValueError(f"[{section}] {key}: expected boolean, got {v!r}")
        if spec.kind == "lower":
            v = v.lower()
            if spec.choices and v not in spec.choices:
                raise ValueError(f"[{section}] {key} must be {_or_list(spec.choices)}")
            if spec.only is not None and v != spec.only:
                raise ValueError(f"current {spec.scope} supports only [{section}] {key}={spec.only}")
        return v


def _fixed10_needs_ten(c: Case) -> None:
    if c.value("run", "run_mode") == "fixed10" and c.value("simple", "max_iterations") != 10:
        raise ValueError("[run] run_mode=fixed10 requires [simple] max_iterations=10")


def _supg_form(c: Case) -> None:
    if not c.value("supg", "enabled"):
        return
    if c.value("supg", "form") != "implicit":
        raise ValueError("current H8 GPU SUPG supports only [supg] form=implicit")
    if c.value("supg", "quad_points") != 64:
        raise ValueError("current H8 GPU SUPG supports only [supg] quad_points=64")


def _single_refresh(c: Case) -> None:
    if c.value("pressure", "fine_csr_refresh_every") != 1:
        raise ValueError("current H8 requires [pressure] fine_csr_refresh_every=1")


def _cheb2_needs_spectrum(c: Case) -> None:
    if c.value("pressure_amg", "smoother") == "cheb2" and c.value("pressure_amg", "spectrum_policy") == "off":
        raise ValueError("[pressure_amg] smoother=cheb2 requires spectrum_policy=auto or always")


CROSS_RULES: Tuple[Callable[[Case], None], ...] = (_fixed10_needs_ten, _supg_form, _single_refresh,
                                                   _cheb2_needs_spectrum)


def command_line(c: Case) -> List[str]:
    """The H8 argv of a case: every flagged key of ``KEYS``, in table order."""
    c.check_names()
    argv: List[str] = []
    for spec in KEYS:
        v = c.value(spec.section, spec.key)  # validates every key, flagged or not
        if spec.flag is None:
            continue
        if spec.kind == "bool":
            v = 1 if v else 0
        argv += [f"--{spec.flag}", str(v)]
    for rule in CROSS_RULES:
        rule(c)
    return argv


def precision_of(c: Case) -> str:
    return c.value("run", "precision")


def find_solver(precision: str, explicit: Optional[str]) -> Path:
    """The executable: --exe, then NODALS_GPU_<PREC>_EXE, then this package's build."""
    tried: List[Path] = []
    if explicit:
        tried.append(Path(os.path.expandvars(os.path.expanduser(explicit))))
    env = os.environ.get(f"NODALS_GPU_{precision.upper()}_EXE")
    if env:
        tried.append(Path(os.path.expandvars(os.path.expanduser(env))))
    tried.append(PACKAGE_LIB / f"nodals_gpu_h8_{precision}")
    usable = [p for p in tried if p.is_file() and os.access(p, os.X_OK)]
    return usable[0] if usable else tried[0]


def stream_to_log(cmd: List[str], log: Path, timeout_s: int) -> int:
    """Run cmd, copying its merged output to stdout and to log line by line;
    EXIT_TIMEOUT when it outlives timeout_s (> 0)."""
    log.parent.mkdir(parents=True, exist_ok=True)
    deadline = None if timeout_s <= 0 else timeout_s
    with log.open("w", encoding="utf-8", errors="replace") as sink, \
            subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, bufsize=1) as proc:
        assert proc.stdout is not None
        for line in proc.stdout:
            sys.stdout.write(line)
            sys.stdout.flush()
            sink.write(line)
            sink.flush()
        try:
            return proc.wait(timeout=deadline)
        except subprocess.TimeoutExpired:
            proc.terminate()
            try:
                proc.wait(5)
            except subprocess.TimeoutExpired:
                proc.kill()
            return EXIT_TIMEOUT


def _passed(log: Path) -> bool:
    for line in log.read_text(encoding="utf-8", errors="replace").splitlines():
        if line.startswith("NODALS_GPU_RESULT gate=H8 ") and "status=PASS" in line:
            return True
    return False


def main(argv: List[str]) -> int:
    argv = list(argv)
    extra: List[str] = []
    if "--" in argv:
        cut = argv.index("--")
        argv, extra = argv[:cut], argv[cut + 1:]
    ap = argparse.ArgumentParser(prog="nodals-gpu", description="Run the B200 SIMPLE solver from a .case file")
    ap.add_argument("case", type=Path)
    ap.add_argument("--dry-run", action="store_true")
    ap.add_argument("--dump-options-json", action="store_true")
    ap.add_argument("--exe", help="solver executable override")
    ap.add_argument("--set", action="append", default=[], metavar="SECTION.KEY=VALUE")
    ns = ap.parse_args(argv)

    path = ns.case.expanduser().resolve()
    c = Case.read(path)
    c.override(ns.set)
    options = command_line(c)
    precision = precision_of(c)
    solver = find_solver(precision, ns.exe)
    name = c.raw("run", "name") or path.stem
    root = str(c.value("run", "output_root"))
    if root.lower() == "auto":
        stamp = datetime.datetime.now().strftime("%Y%m%d_%H%M%S")
        outroot = Path.home() / "Downloads" / f"NodalS_GPU_{name}_{stamp}"
    else:
        outroot = Path(os.path.expandvars(os.path.expanduser(root)))
    log = outroot / f"{name}.log"
    cmd = [str(solver), *options, *extra]

    print(f"NODALS_GPU_CASE name={name} file={path} precision={precision} output={outroot}")
    print("NODALS_GPU_COMMAND " + shlex.join(cmd))
    if ns.dump_options_json:
        print("NODALS_GPU_OPTIONS_JSON=" + json.dumps(options))
    if ns.dry_run:
        print("NODALS_GPU_CASE_RESULT status=DRY_RUN")
        return EXIT_PASS
    if not (solver.is_file() and os.access(solver, os.X_OK)):
        print(f"NODALS_GPU_CASE_RESULT status=FAIL reason=missing_solver executable={solver}", file=sys.stderr)
        return EXIT_NO_SOLVER
    rc = stream_to_log(cmd, log, int(c.value("run", "timeout_seconds")))
    print(f"NODALS_GPU_ARTIFACTS log={log} outroot={outroot}")
    if rc != 0:
        print(f"NODALS_GPU_CASE_RESULT status=FAIL rc={rc}")
        return rc
    if _passed(log):
        print("NODALS_GPU_CASE_RESULT status=PASS")
        return EXIT_PASS
    print("NODALS_GPU_CASE_RESULT status=NOT_CONVERGED reason=no_NODALS_GPU_RESULT_PASS")
    return EXIT_NOT_CONVERGED


def cli() -> int:
    try:
        return main(sys.argv[1:])
    except (ValueError, configparser.Error, OSError) as e:
        print(f"NODALS_GPU_CASE_ERROR {e}", file=sys.stderr)
        return EXIT_CONFIG


if __name__ == "__main__":
    raise SystemExit(cli())
