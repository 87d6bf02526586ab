"""The .case front end end to end on a GPU: the annotated case file, pointed
at a small seeded pipe and switched to the fixed ten-iteration run mode,
runs the drop-in executable and reports PASS (exit 0), with the solver log in
the output root; the same with laminar SUPG switched on."""
from __future__ import annotations

import subprocess
import sys

import pytest

from conftest import ROOT

CASE = ROOT / "nodals_b200" / "cases" / "gpu-h8-annotated.case"


@pytest.mark.gpu
@pytest.mark.parametrize("extra", [[], ["--set", "supg.enabled=true"]], ids=["plain", "supg"])
def test_annotated_case_runs(meshes, tmp_path, extra):
    from nodals_b200 import meshgen
    msh = tmp_path / "pipe.msh"
    meshgen.write_msh2(meshes("pipe_small"), str(msh))
    out = tmp_path / "out"
    sets = ["--set", f"solver.mesh={msh}", "--set", f"run.output_root={out}", "--set", "run.run_mode=fixed10",
            "--set", "simple.max_iterations=10", "--set", "run.precision=fp64",
            "--set", "pressure_amg.terminal_rows=100"]
    r = subprocess.run([sys.executable, "-m", "nodals_b200.case", str(CASE), *sets, *extra], cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "NODALS_GPU_CASE_RESULT status=PASS" in r.stdout
    logs = list(out.glob("*.log"))
    assert len(logs) == 1
    text = logs[0].read_text()
    assert text.count("NODALS_GPU_H8_SIMPLE") >= 10
    assert ("NODALS_GPU_H8_SUPG" in text) == bool(extra)
