"""The drop-in executable end to end on a GPU: the same command line as the
reference binary run that produced each fixture (tests/golden/run_*.npz),
given to nodals_b200/_lib/nodals_gpu_h8_{fp64,fp32}.  The NODALS_GPU_H8_SIMPLE
lines must carry the reference's relCont (1e-8 relative; SUPG 1e-7; FP32
2e-3) and pressure iteration counts (FP64), the exit code must match, and the
VTU written by --vtu-out must hold the reference's P0 pressure and
cell-average velocity (1e-8 relative L2; FP32 1e-3)."""
from __future__ import annotations

import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, rel_l2
from test_gpu_parity import SUPG_TOL

sys.path.insert(0, str(GOLDEN))
import make_golden  # noqa: E402

LIB = ROOT / "nodals_b200" / "_lib"
MESH = {"tiny": "pipe_tiny", "small": "pipe_small", "m40k": "pipe40k"}


def _cases():
    return sorted(p.stem[4:] for p in GOLDEN.glob("run_*.npz"))


@pytest.mark.gpu
@pytest.mark.parametrize("case", _cases())
def test_executable_reproduces_reference_run(case, tmp_path):
    g = np.load(GOLDEN / f"run_{case}.npz")
    toks = str(g["cmd"]).split()
    # drop the reference's own output path; ours goes to tmp_path
    args, i = [], 0
    while i < len(toks):
        if toks[i] == "--vtu-out":
            i += 2
            continue
        args.append(toks[i])
        i += 1
    supg = "--supg" in args
    fp32 = case.endswith("fp32")
    mesh = make_golden.write_mesh(MESH[case.split("_")[0]], tmp_path)
    vtu = tmp_path / "out.vtu"
    exe = LIB / ("nodals_gpu_h8_fp32" if fp32 else "nodals_gpu_h8_fp64")
    cmd = [str(exe), "--mesh", str(mesh), *args, "--vtu-out", str(vtu)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == int(g["rc"][0]), (r.returncode, r.stderr[-2000:])
    assert re.search(r"NODALS_GPU_RESULT gate=H8 .*status=(PASS|FAIL)", r.stdout)
    its, rel, pcg, _, _ = make_golden.parse_log(r.stdout)
    want = {int(i): k for k, i in enumerate(g["it"])}
    got = {int(i): k for k, i in enumerate(its)}
    assert set(want) <= set(got), (sorted(want), sorted(got))
    tol = 2e-3 if fp32 else (SUPG_TOL if supg else 1e-8)
    for it, k in want.items():
        j = got[it]
        assert abs(rel[j] - g["rel_cont"][k]) <= tol * abs(g["rel_cont"][k]) + 1e-12, (it, rel[j], g["rel_cont"][k])
        if not fp32:
            assert pcg[j] == int(g["p_its"][k]), (it, pcg[j], int(g["p_its"][k]))
    if "p" in g.files:
        p, u0 = make_golden.parse_vtu(vtu)
        ftol = 1e-3 if fp32 else 1e-8
        assert rel_l2(p, g["p"]) <= ftol
        assert rel_l2(u0, g["u_cell"]) <= ftol


@pytest.mark.gpu
def test_executable_reads_hxt1(tmp_path):
    """--mesh given the HXT1 file the reference's converter made from the
    pipe_tiny mesh: every NODALS_GPU_H8_SIMPLE line equals the one of the
    MSH 2.2 run of the same mesh."""
    from nodals_b200 import meshgen
    msh = meshgen.write_msh2(meshgen.named("pipe_tiny"), tmp_path / "m.msh")
    exe = LIB / "nodals_gpu_h8_fp64"
    common = ["--run-mode", "fixed10", "--max-outer", "10", "--amg-terminal", "60", "--p-rtol", "1e-6", "--p-max", "200"]
    outs = []
    for mesh in (msh, GOLDEN / "hxt1_pipe_tiny.bin"):
        r = subprocess.run([str(exe), "--mesh", str(mesh), *common], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append([l for l in r.stdout.splitlines() if l.startswith("NODALS_GPU_H8_SIMPLE")])
    assert len(outs[0]) == 10 and outs[0] == outs[1]
