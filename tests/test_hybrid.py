"""Mixed hexahedron/tetrahedron solvers against the reference binaries' own
runs on the same HXT1 mesh: the Stokes gate (the reference's HXT4A,
gpu/serial_cuda/hybrid_hxt4a/hxt4a_main.cu) against the reference binary's
own run on the same HXT1 mesh (tests/golden/hxt4a_hybrid_r2.log, made by
make_hxt4a_golden.py from tests/golden/hxt1_hybrid_r2.bin, itself the
reference preparer's output for the seeded 2-ring hybrid pipe).

CPU: the host-assembled operators (hex Q1+BF2 diffusion, tet P1+BF3
diffusion, Nitsche interface, divergence with averaged interface traces,
rAU) reproduce the reference's printed operator-audit norms to 1e-12.
GPU: the gate executable prints the same audit, the same relCont history
(1e-9 relative; the reference sums with atomics, so not bitwise), CG counts
within one iteration, the same outer iteration count and the same result
line (errors against p* and the Hagen-Poiseuille-like checks 1e-8).

The mixed-mesh pipe SIMPLE (the reference's HXT4B,
gpu/serial_cuda/hybrid_hxt4b/hxt4b_main.cu; logs made by
make_hxt4b_golden.py): with tight pressure solves every printed iteration,
the converged iteration and the physics line agree with the reference to
3e-9.  At the default pressure tolerance (rtol 0.9) the iteration amplifies
rounding -- the reference's own runs differ from each other, its atomic
sums changing the last bits -- so there the first iteration agrees to 1e-10,
the converged iteration within 5 and the physics within 5e-3.

The VTU of --vtu (hxt4b_main.cu:203-209): on the CPU the C-ABI writer, given
seeded fields, produces byte for byte the text of the oracle's restatement
of the reference writer; on the GPU the tight run's file has the reference
run's layout and integer blocks exactly and its values to 3e-9 of each
block's largest magnitude (tests/golden/hxt4b_hybrid_r2_tight.vtu.gz).

The AMG-preconditioned pressure solve (--pressure-solver pcg_amg, the
preconditioner of the reference's turbulent entry) with tight pressure
solves follows the same tight history with a fifth of the pressure
iterations or fewer; the reference's own cheb2 V-cycle makes PCG break down on this
matrix and the run fails as the reference's would.
"""
from __future__ import annotations

import ctypes as C
import gzip
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from oracle import hybrid_vtu

MESH = GOLDEN / "hxt1_hybrid_r2.bin"
LOG = GOLDEN / "hxt4a_hybrid_r2.log"


def _kv(line):
    return dict(re.findall(r"(\w+)=(\[[^\]]*\]|\S+)", line))


def _parse(text):
    lines = text.splitlines()
    audit = next(_kv(l) for l in lines if l.startswith("NODALS_HXT4A_OPERATOR_AUDIT"))
    simple = {int(_kv(l)["it"]): _kv(l) for l in lines if l.startswith("NODALS_HXT4A_SIMPLE")}
    result = next(_kv(l) for l in lines if l.startswith("NODALS_HXT4A_RESULT"))
    return audit, simple, result


def _close(a, b, tol):
    a, b = float(a), float(b)
    return abs(a - b) <= tol * max(abs(b), 1e-300)


def test_host_operators_match_reference_audit(native):
    audit, _, _ = _parse(LOG.read_text())
    n = (C.c_double * 3)()
    rc = native.lib().nds_hybrid_operator_audit(str(MESH).encode(), C.c_double(1.0), C.c_double(50.0), C.c_double(24.0), n)
    assert rc == 0, native.lib().nds_last_error()
    for got, key in zip(n, ("Anorm", "Bnorm", "Snorm")):
        assert _close(got, audit[key], 1e-12), (key, got, audit[key])


@pytest.mark.gpu
def test_gate_matches_reference_run():
    r = subprocess.run([str(ROOT / "nodals_b200" / "_lib" / "nodals_hxt4a_fp64"), "--mesh", str(MESH)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "HXT4A_PRECISION_STATUS=PASS" in r.stdout
    ga, gs, gr = _parse(r.stdout)
    wa, ws, wr = _parse(LOG.read_text())
    for k in ("Anorm", "Bnorm", "Snorm"):
        assert _close(ga[k], wa[k], 1e-12), (k, ga[k], wa[k])
    assert sorted(gs) == sorted(ws)
    for it, w in ws.items():
        g = gs[it]
        assert _close(g["relCont"], w["relCont"], 1e-9), (it, g["relCont"], w["relCont"])
        assert _close(g["velocityNorm"], w["velocityNorm"], 1e-9), (it, g["velocityNorm"], w["velocityNorm"])
        gm, wm = eval(g["mCG"]), eval(w["mCG"])
        assert all(abs(x - y) <= 1 for x, y in zip(gm, wm)) and abs(int(g["pCG"]) - int(w["pCG"])) <= 1, (it, g, w)
    assert gr["outer"] == wr["outer"]
    for k, tol in (("finalRelCont", 1e-9), ("pressureRelL2", 1e-8), ("slope", 1e-10), ("delta", 1e-10),
                   ("velocityRel", 1e-8)):
        assert _close(gr[k], wr[k], tol), (k, gr[k], wr[k])
    assert abs(float(gr["avgMomentumCG"]) - float(wr["avgMomentumCG"])) < 0.01
    assert abs(float(gr["avgPressureCG"]) - float(wr["avgPressureCG"])) < 0.01


def _parse_4b(text):
    lines = text.splitlines()
    simple = {int(_kv(l)["it"]): _kv(l) for l in lines if l.startswith("NODALS_HXT4B_SIMPLE")}
    phys = next(_kv(l) for l in lines if l.startswith("NODALS_HXT4B_PHYSICS"))
    cfg = next(_kv(l) for l in lines if l.startswith("NODALS_HXT4B_CONFIG"))
    cfg.update(next(_kv(l) for l in lines if l.startswith("NODALS_HXT4B_HAGEN_POISEUILLE")))
    return cfg, simple, phys


def test_vtu_writer_matches_reference_layout(native, tmp_path):
    m = hybrid_vtu.read_mixed_hxt1(MESH)
    counts = (C.c_uint64 * 13)()
    assert native.lib().nds_hybrid_counts(str(MESH).encode(), counts) == 0
    assert tuple(counts) == tuple(m["counts"])
    nvel, npr = int(counts[5]), int(counts[6])
    rng = np.random.default_rng(7)
    u = [rng.standard_normal(nvel) * 10.0 ** rng.integers(-12, 3, nvel) for _ in range(3)]
    p = rng.standard_normal(npr) * 16.0
    out = tmp_path / "seeded.vtu"
    dp = C.POINTER(C.c_double)
    args = [np.ascontiguousarray(a).ctypes.data_as(dp) for a in (*u, p)]
    assert native.lib().nds_hybrid_write_vtu(str(MESH).encode(), str(out).encode(), *args) == 0
    assert out.read_text() == hybrid_vtu.vtu_text(m, *u, p)
    assert native.lib().nds_hybrid_write_vtu(str(MESH).encode(), str(tmp_path / "no" / "x.vtu").encode(), *args) != 0


def _same_vtu(got: str, want: str, tol: float):
    number = re.compile(r"(?<=\n)[-+0-9.eE ]+(?=\n)")
    assert number.sub("#", got) == number.sub("#", want)
    g, w = hybrid_vtu.parse_vtu(got), hybrid_vtu.parse_vtu(want)
    assert sorted(g) == sorted(w)
    for name in ("points", "connectivity", "offsets", "types", "region"):
        assert np.array_equal(g[name], w[name]), name
    for name in ("velocity_Q1P1_vertex", "pressure_Q0P0_vertex_volume_average", "pressure_Q0P0"):
        scale = np.abs(w[name]).max()
        err = np.abs(g[name] - w[name]).max()
        assert err <= tol * scale, (name, err, scale)


def _run_4b(vtu, *extra):
    r = subprocess.run([str(ROOT / "nodals_b200" / "_lib" / "nodals_hxt4b_fp64"), "--mesh", str(MESH), "--vtu", str(vtu),
                        *extra], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "HXT4B_GATE_STATUS=PASS" in r.stdout
    assert f"NODALS_HXT4B_OUTPUT vtu={vtu} status=PASS" in r.stdout
    return _parse_4b(r.stdout)


PHYS = ("pressureSlope", "pIn", "pOut", "pressureDrop", "vertexVelocityProfileRelL2", "transverseVertexRelL2",
        "convectionActionNorm", "velocityNorm")


@pytest.mark.gpu
def test_pipe_simple_matches_reference_tight(tmp_path):
    vtu = tmp_path / "r2.vtu"
    gc, gs, gp = _run_4b(vtu, "--p-rtol", "1e-10", "--p-max", "2000")
    wc, ws, wp = _parse_4b((GOLDEN / "hxt4b_hybrid_r2_tight.log").read_text())
    for k in ("cellsHex", "cellsTet", "velocityDofs", "pressureDofs", "csrNnz", "colors", "maxColor", "pressureGaugePin"):
        assert gc.get(k) == wc.get(k), k
    assert sorted(gs) == sorted(ws)
    for it, w in ws.items():
        g = gs[it]
        for k in ("relCont", "absCont", "zMomentumResidualRel"):
            assert _close(g[k], w[k], 3e-9), (it, k, g[k], w[k])
        assert abs(int(g["pCG"]) - int(w["pCG"])) <= 1, (it, g["pCG"], w["pCG"])
    for k in PHYS:
        assert _close(gp[k], wp[k], 3e-9), (k, gp[k], wp[k])
    _same_vtu(vtu.read_text(), gzip.decompress((GOLDEN / "hxt4b_hybrid_r2_tight.vtu.gz").read_bytes()).decode(), 3e-9)


@pytest.mark.gpu
def test_pipe_simple_default_tolerance(tmp_path):
    gc, gs, gp = _run_4b(tmp_path / "r2.vtu", "--p-max", "400")
    wc, ws, wp = _parse_4b((GOLDEN / "hxt4b_hybrid_r2.log").read_text())
    for k in ("relCont", "absCont", "zMomentumResidualRel"):
        assert _close(gs[1][k], ws[1][k], 1e-10), (k, gs[1][k], ws[1][k])
    assert abs(max(gs) - max(ws)) <= 5, (max(gs), max(ws))
    for k in PHYS:
        assert _close(gp[k], wp[k], 5e-3), (k, gp[k], wp[k])


AMG = ["--pressure-solver", "pcg_amg"]
AMG_VARIANTS = {"cheb2_separate_post": AMG + ["--amg-separate-post", "1"], "mcgs": AMG + ["--amg-smoother", "mcgs"]}


@pytest.mark.gpu
@pytest.mark.parametrize("variant", sorted(AMG_VARIANTS))
def test_pipe_simple_amg_pressure_tight(tmp_path, variant):
    """With tight pressure solves the SIMPLE iterates do not depend on the
    pressure preconditioner: the AMG-preconditioned runs follow the
    reference's (Jacobi-preconditioned) tight history to 3e-9, with a fifth
    of its pressure iterations or fewer."""
    gc, gs, gp = _run_4b(tmp_path / "r2.vtu", "--p-rtol", "1e-10", "--p-max", "400", *AMG_VARIANTS[variant])
    wc, ws, wp = _parse_4b((GOLDEN / "hxt4b_hybrid_r2_tight.log").read_text())
    assert gc["pressureSolver"] == "PCG_AMG"
    assert sorted(gs) == sorted(ws)
    for it, w in ws.items():
        for k in ("relCont", "absCont", "zMomentumResidualRel"):
            assert _close(gs[it][k], w[k], 3e-9), (it, k, gs[it][k], w[k])
        assert int(gs[it]["pCG"]) * 5 <= int(w["pCG"]), (it, gs[it]["pCG"], w["pCG"])
    for k in PHYS:
        assert _close(gp[k], wp[k], 3e-9), (k, gp[k], wp[k])


@pytest.mark.gpu
def test_pipe_simple_reference_cheb2_vcycle_breaks_pcg(tmp_path):
    """The reference's cheb2 V-cycle (post-smoothing aliasing) is not a
    positive definite preconditioner of this pressure matrix: PCG reports a
    nonpositive rho and the executable exits 2, as the reference's pcg_amg
    throws."""
    r = subprocess.run([str(ROOT / "nodals_b200" / "_lib" / "nodals_hxt4b_fp64"), "--mesh", str(MESH), "--vtu",
                        str(tmp_path / "x.vtu"), "--p-max", "400", *AMG], capture_output=True, text=True, timeout=600)
    assert r.returncode == 2
    assert "nonpositive" in r.stderr and "HXT4B_GATE_STATUS=FAIL" in r.stderr


def test_operator_patch_matches_reference_hxt2_gate(native):
    """The velocity operator without boundary conditions (nu 1, gamma 20)
    against the reference's HXT2 gate run on the same mesh
    (tests/golden/hxt2_hybrid_r2.log, made by make_hxt2_golden.py): the
    volume-only residual of each affine field at the interface bubbles and
    the energies x.Ax, y.Ay, x.Ay, y.Ax to 1e-11 (12 printed digits); the
    gate's own criteria for the round-off quantities (constant patch below
    1e-11, Nitsche cancelling the affine interface residual to 1e-7 of it,
    symmetry)."""
    lines = (GOLDEN / "hxt2_hybrid_r2.log").read_text().splitlines()
    aff = [_kv(l) for l in lines if l.startswith("NODALS_HXT2_AFFINE_PATCH")]
    sym = next(_kv(l) for l in lines if l.startswith("NODALS_HXT2_SYMMETRY_ENERGY"))
    out = (C.c_double * 12)()
    assert native.lib().nds_hybrid_operator_patch(str(MESH).encode(), C.c_double(1.0), C.c_double(20.0), out) == 0
    assert out[0] < 1e-11
    for k, a in enumerate(aff):
        assert _close(out[1 + k], a["volumeInterfaceBubbleMax"], 1e-11), (k, out[1 + k], a)
        assert out[4 + k] < 1e-7 * out[1 + k]
    for i, key in enumerate(("xAx", "yAy", "xAy", "yAx")):
        assert _close(out[7 + i], sym[key], 1e-11), (key, out[7 + i], sym[key])
    assert int(out[11]) == int(sym["interfaceBubbleDofs"])
    assert abs(out[9] - out[10]) <= 1e-12 * abs(out[9])


def test_divergence_audit_matches_reference_hxt3a_gate(native):
    """The divergence B of the mixed mesh against the reference's HXT3A gate
    run on the same mesh (tests/golden/hxt3a_hybrid_r2.log, made by
    make_hxt3a_golden.py): the nonzero count exactly, p.Bu, u.B^T p, the four
    Schur energies, the cross-region trace norms and direct Schur entries to
    1e-11; the round-off quantities (constant and affine divergence) within
    1e-15.  (The reference gate itself reports FAIL on this mesh: its
    constant-divergence bound of 2e-18 is below the 4.9e-17 round-off that
    both codes give.)"""
    kv = {}
    for l in (GOLDEN / "hxt3a_hybrid_r2.log").read_text().splitlines():
        if l.startswith("NODALS_HXT3A_"):
            kv[l.split()[0]] = _kv(l)
    out = (C.c_double * 16)()
    assert native.lib().nds_hybrid_divergence_audit(str(MESH).encode(), out) == 0
    assert int(out[0]) == int(kv["NODALS_HXT3A_BCSR"]["nnz"])
    assert abs(out[1] - float(kv["NODALS_HXT3A_CONSTANT_DIVERGENCE"]["cellResidualMax"])) < 1e-15
    aff = kv["NODALS_HXT3A_AFFINE_DIVERGENCE"]
    assert abs(out[2] - float(aff["maxAbs"])) < 1e-15 and out[3] < 2e-10
    t = kv["NODALS_HXT3A_TRANSPOSE"]
    assert _close(out[4], t["pDotBu"], 1e-11) and _close(out[5], t["uDotBTp"], 1e-11)
    sc = kv["NODALS_HXT3A_SCHUR"]
    for i, key in enumerate(("xSx", "ySy", "xSy", "ySx")):
        assert _close(out[6 + i], sc[key], 1e-11), (key, out[6 + i], sc[key])
    s = kv["NODALS_HXT3A_INTERFACE_SENSITIVITY"]
    for i, key in enumerate(("crossCoeffNormMin", "crossCoeffNormMax", "directSchurAbsMin", "directSchurAbsMax")):
        assert _close(out[10 + i], s[key], 1e-11), (key, out[10 + i], s[key])
    assert int(out[14]) == int(s["trianglePairs"]) and int(out[15]) == 0


def _oracle_history(native, n, **opts):
    from oracle.hybrid_flow import HybridFlowOracle
    return HybridFlowOracle(native, MESH, **opts).run(n)


def test_flow_oracle_matches_reference_tight(native):
    """The CPU restatement of the mixed-mesh pipe SIMPLE (oracle/hybrid_flow.py)
    on the product's host setup follows the reference's tight run: relCont
    and absCont of the first five iterations to 1e-11, the same pressure
    iteration counts."""
    hist = _oracle_history(native, 5, p_rtol=1e-10, p_max=2000)
    _, ws, _ = _parse_4b((GOLDEN / "hxt4b_hybrid_r2_tight.log").read_text())
    for it in range(1, 6):
        rel, cn, its = hist[it - 1]
        assert _close(rel, ws[it]["relCont"], 1e-11), (it, rel, ws[it]["relCont"])
        assert _close(cn, ws[it]["absCont"], 1e-11), (it, cn, ws[it]["absCont"])
        assert its == int(ws[it]["pCG"]), (it, its, ws[it]["pCG"])


@pytest.mark.gpu
def test_pipe_simple_device_matches_oracle(native, tmp_path):
    """The device run against the oracle on the same host setup: the first
    five iterations' relCont and absCont to 3e-9, pressure iterations within
    one (tight pressure solves)."""
    _, gs, _ = _run_4b(tmp_path / "r2.vtu", "--p-rtol", "1e-10", "--p-max", "2000")
    hist = _oracle_history(native, 5, p_rtol=1e-10, p_max=2000)
    for it in range(1, 6):
        rel, cn, its = hist[it - 1]
        assert _close(gs[it]["relCont"], rel, 3e-9), (it, gs[it]["relCont"], rel)
        assert _close(gs[it]["absCont"], cn, 3e-9), (it, gs[it]["absCont"], cn)
        assert abs(int(gs[it]["pCG"]) - its) <= 1, (it, gs[it]["pCG"], its)


def test_flow_setup_properties(native):
    """Host setup of the pipe SIMPLE: no two rows of a colour are coupled (so a
    colour's rows update independently), fixed rows are in no colour, every
    local convection value is gathered into exactly one entry, and each
    diagonal position points at the row's own column."""
    import numpy as np
    h = native.HybridAmg(MESH, None)
    row, col, dpos = h.array("flow.row"), h.array("flow.col"), h.array("flow.diagPos")
    n = len(row) - 1
    assert np.array_equal(col[dpos], np.arange(n))
    off, rows = h.array("flow.colourOff"), h.array("flow.colourRows")
    fixed = h.array("flow.fixed").astype(bool)
    colour = np.full(n, -1)
    for c in range(len(off) - 1):
        colour[rows[off[c]:off[c + 1]]] = c
    assert np.all((colour >= 0) == ~fixed)
    r_of = np.repeat(np.arange(n), np.diff(row))
    coupled = (r_of != col) & (colour[r_of] >= 0) & (colour[r_of] == colour[col])
    assert not coupled.any()
    src, soff = h.array("flow.src"), h.array("flow.srcOff")
    sc = h.array("flow.scalars")
    assert np.array_equal(np.sort(src), np.arange(int(sc[5]) * 196 + int(sc[6]) * 64))
    assert soff[-1] == len(src) and len(soff) == len(col) + 1
