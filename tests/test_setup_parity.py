"""Host setup parity against the reference's own setup builders.

Fixtures tests/golden/setup_*.npz were written by oracle/_ref/ref_setup_dump
(the reference's load_foam_tet_mesh, build_g4_setup, build_h2_fine_csr_host,
build_sa_hierarchy / build_cf_hierarchy compiled from the reference tree).
Integer arrays (numbering, colouring, cell plans, fine CSR topology,
aggregates, transfer and coarse patterns) must be bit-exact; floating arrays
agree to round-off (<= 1e-12 relative to the array's max magnitude; the
quadrature here is computed, the reference's is a 17-digit table).
When the reference tree and oracle/_ref are present, the same comparison is
also made directly on larger meshes.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, REFERENCE, ROOT

FLOAT_TOL = 1e-12
CASES = {
    "tiny_sa": dict(amg_hierarchy="sa", amg_terminal=60, re=20.0, alpha_u=0.7),
    "tiny_cf": dict(amg_hierarchy="cf", cf_pmax=8, cf_interp="exti", amg_terminal=60, re=20.0, alpha_u=0.7,
                    amg_smoother="jacobi"),
}


def compare(P, ref: dict, skip=()):
    bad = []
    for k, v in ref.items():
        if k in skip:
            continue
        if k in ("amg.levels",):
            assert int(P.scalar(k)) == int(v[0])
            continue
        mine = P.array(k)
        if k.endswith("nCoarse"):
            assert int(mine[0]) == int(v[0]), k
            continue
        assert mine.shape == v.shape, (k, mine.shape, v.shape)
        if v.dtype.kind in "iu":
            if not np.array_equal(mine, v):
                bad.append((k, int(np.count_nonzero(mine != v))))
        elif v.size:
            err = float(np.max(np.abs(mine - v)) / max(np.max(np.abs(v)), 1e-300))
            if not err <= FLOAT_TOL:
                bad.append((k, err))
    assert not bad, bad


@pytest.mark.parametrize("case", sorted(CASES))
def test_setup_matches_reference_fixture(native, meshes, case):
    ref = dict(np.load(GOLDEN / f"setup_{case}.npz"))
    m = native.Mesh.from_tetmesh(meshes("pipe_tiny"))
    P = native.Problem(m, max_outer=10, **CASES[case])
    compare(P, ref)


def test_polymesh_msh2_and_arrays_agree(native, meshes, tmp_path):
    from nodals_b200 import meshgen
    tm = meshes("pipe_tiny")
    pm = meshgen.write_polymesh(tm, tmp_path / "pm")
    msh = meshgen.write_msh2(tm, tmp_path / "m.msh")
    probs = [native.Problem(native.Mesh.read_polymesh(pm), max_outer=10),
             native.Problem(native.Mesh.read_msh2(msh), max_outer=10),
             native.Problem(native.Mesh.from_tetmesh(tm), max_outer=10)]
    for k in ("mesh.tets", "mesh.opp_face", "g2free", "mom.col", "color", "cell.ref", "cell.rowSlot", "fine.col",
              "amg.agg0", "amg.P0.col"):
        for P in probs[1:]:
            assert np.array_equal(probs[0].array(k), P.array(k)), k
    for k in ("mom.val", "initRau", "amg.A0.val", "fixedValue"):
        for P in probs[1:]:
            assert np.array_equal(probs[0].array(k), P.array(k)), k


def test_setup_is_deterministic(native, meshes):
    m = native.Mesh.from_tetmesh(meshes("pipe_small"))
    a = native.Problem(m, max_outer=10, amg_hierarchy="cf", amg_smoother="jacobi", cf_interp="exti", cf_pmax=8)
    b = native.Problem(m, max_outer=10, amg_hierarchy="cf", amg_smoother="jacobi", cf_interp="exti", cf_pmax=8)
    for k in ("color", "fine.col", "amg.P0.col", "amg.P0.val", "amg.A0.val", "amg.terminal_inv"):
        assert np.array_equal(a.array(k), b.array(k)), k


def test_invalid_options_rejected(native, meshes):
    m = native.Mesh.from_tetmesh(meshes("pipe_tiny"))
    with pytest.raises(native.NdsError, match="fixed10 requires maxOuter=10"):
        native.Problem(m)                                   # binary defaults: fixed10 with 2500 outer
    with pytest.raises(native.NdsError, match="cf-pmax"):
        native.Problem(m, max_outer=10, cf_pmax=0)
    with pytest.raises(native.NdsError, match="Chebyshev AMG smoother requires spectrum"):
        native.Problem(m, max_outer=10, amg_spectrum_policy="off")
    with pytest.raises(native.NdsError, match="patch not found"):
        native.Problem(m, max_outer=10, wall="nope")


def _ref_dump_available():
    return (ROOT / "oracle" / "_ref" / "ref_setup_dump").exists() and REFERENCE is not None


@pytest.mark.skipif(not _ref_dump_available(), reason="reference tree / oracle/_ref not present")
@pytest.mark.parametrize("mesh,flags,opts", [
    ("pipe_small", ["--amg-hierarchy", "sa", "--amg-terminal", "100", "--alpha-u", "0.7"],
     dict(amg_hierarchy="sa", amg_terminal=100, alpha_u=0.7)),
    ("pipe_small", ["--amg-hierarchy", "cf", "--cf-pmax", "4", "--cf-interp", "direct", "--power-its", "16"],
     dict(amg_hierarchy="cf", cf_pmax=4, cf_interp="direct", amg_smoother="cheb2")),
    ("reference40k", ["--amg-hierarchy", "sa", "--alpha-u", "0.5"], dict(amg_hierarchy="sa", alpha_u=0.5)),
    # the SUPG entry: its setup snapshot includes the SUPG terms of the
    # convecting Dirichlet values (h8_supg_main_setup.inc:6-7)
    ("pipe_small", ["--amg-hierarchy", "sa", "--amg-terminal", "100", "--alpha-u", "0.7", "--supg", "1"],
     dict(amg_hierarchy="sa", amg_terminal=100, alpha_u=0.7, supg=1)),
    ("pipe_small", ["--amg-hierarchy", "cf", "--cf-pmax", "8", "--cf-interp", "exti", "--power-its", "16", "--supg", "1",
                    "--supg-tau-scale", "0.1", "--supg-magic", "4"],
     dict(amg_hierarchy="cf", cf_pmax=8, cf_interp="exti", amg_smoother="cheb2", supg=1, supg_tau_scale=0.1,
          supg_magic=4.0)),
])
def test_setup_matches_reference_builders_directly(native, meshes, tmp_path, mesh, flags, opts):
    from nodals_b200 import meshgen
    from oracle.dump import read_dump
    if mesh == "reference40k":
        pm = REFERENCE / "meshes" / "pipe" / "40k" / "constant" / "polyMesh"
    else:
        pm = meshgen.write_polymesh(meshes(mesh), tmp_path / mesh)
    dump = tmp_path / "d.bin"
    subprocess.run([str(ROOT / "oracle" / "_ref" / "ref_setup_dump"), "--mesh", str(pm), "--out", str(dump), *flags],
                   check=True, stdout=subprocess.DEVNULL)
    ref = read_dump(dump)
    P = native.Problem(native.Mesh.read_polymesh(pm), max_outer=10, **opts)
    compare(P, ref, skip=("mesh.face_patch", "fixedSlot", "cell.invJ", "initDelta", "pipe.R", "pipe.L"))
