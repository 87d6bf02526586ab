"""Argument handling of the drop-in executable on CPU: reference messages on
stderr (NODALS_GPU_H8_EXCEPTION) and exit code 90 for rejected controls,
before any device work."""
from __future__ import annotations

import subprocess

import pytest

from conftest import ROOT

EXE = ROOT / "nodals_b200" / "_lib" / "nodals_gpu_h8_fp64"


@pytest.fixture(scope="module")
def msh(native, meshes, tmp_path_factory):
    from nodals_b200 import meshgen
    p = tmp_path_factory.mktemp("cli") / "tiny.msh"
    meshgen.write_msh2(meshes("pipe_tiny"), str(p))
    return p


def _run(*args):
    return subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("flags,message", [
    (["--supg", "1", "--supg-form", "explicit"], "H8 GPU SUPG currently supports form=implicit"),
    (["--supg", "1", "--supg-quad-points", "27"], "H8 GPU SUPG currently supports quad-points=64"),
    (["--supg", "1", "--supg-tau-scale", "0"], "H8 SUPG tau scale must be positive"),
    (["--supg", "1", "--momentum-work", "sgs1", "--run-mode", "fixed10", "--max-outer", "10"],
     "H8 requires momentum-work=fgs1"),
    (["--no-such-flag", "1"], "H8 usage error"),
    (["--run-mode", "fixed10", "--max-outer", "11"], "H8 fixed10 requires maxOuter=10"),
])
def test_rejected_controls(msh, flags, message):
    r = _run("--mesh", msh, *flags)
    assert r.returncode == 90, (r.returncode, r.stdout[-500:], r.stderr[-500:])
    assert "NODALS_GPU_H8_EXCEPTION" in r.stderr and message in r.stderr
