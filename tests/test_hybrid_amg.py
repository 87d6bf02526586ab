"""Setup of the mixed-mesh pressure preconditioner against the reference's own
builders (hxt4c::build_hybrid_fine_host, hybrid_hxt5b/hybrid_amg.cuh:63, and
build_cf_hierarchy_from_csr, hybrid_cf_overload.inc:5), run on the same HXT1
mesh and rAU by oracle/ref_hybrid_amg_dump (tests/golden/hybrid_amg_r2.npz,
made by make_hybrid_amg_golden.py).

The pressure matrix B diag(rAU) B^T (pin row identity, pin column dropped):
pattern, entry rows and diagonal positions identical, values to 1e-12 of the
largest.  The CF hierarchy (PMIS split, extended+i or direct interpolation
with pruning, aggressive first stage, Galerkin products, spectrum estimates,
terminal inverse): every index array identical, values to 1e-12.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

MESH = GOLDEN / "hxt1_hybrid_r2.bin"
GOLD = GOLDEN / "hybrid_amg_r2.npz"
CASES = {
    "exti_t60": dict(amg_terminal=60),
    "direct_aggr_t40": dict(amg_terminal=40, cf_interp=0, cf_aggressive_first=1, cf_pmax=4, cf_theta=0.3),
}


def _rau(nvel):
    g = np.arange(nvel, dtype=np.float64)
    return 0.02 * (1.5 + np.sin(0.37 * (g + 1)))


def _same(name, got, want):
    assert got.shape == want.shape, (name, got.shape, want.shape)
    if want.dtype.kind == "f":
        scale = max(float(np.abs(want).max()), 1e-300) if want.size else 1.0
        assert float(np.abs(got - want).max(initial=0.0)) <= 1e-12 * scale, name
    else:
        assert np.array_equal(got.astype(np.int64), want.astype(np.int64)), name


@pytest.mark.parametrize("case", sorted(CASES))
def test_pressure_hierarchy_matches_reference_builders(native, case):
    z = np.load(GOLD)
    want = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(case + "/")}
    nvel = native.hybrid_counts(MESH)[5]
    h = native.HybridAmg(MESH, _rau(nvel), pressure_solver=1, **CASES[case])
    levels = int(want["amg.levels"][0])
    assert int(h.array("amg.levels")[0]) == levels
    assert int(h.array("pin")[0]) == int(want["pin"][0])
    names = [k for k in want if k not in ("amg.levels", "pin")]
    assert any(k.startswith("amg.P") for k in names)
    for k in names:
        _same(k, h.array(k), want[k])
    if case == "exti_t60":
        assert {"fine.row", "fine.col", "fine.val", "fine.entryRow", "fine.diagPos"} <= set(names)


@pytest.mark.parametrize("bad", [dict(amg_smoother=3, amg_mcgs_order=1), dict(amg_spectrum_policy=2),
                                 dict(cf_interp=7), dict(amg_terminal=0)])
def test_pressure_options_rejected(native, bad):
    nvel = native.hybrid_counts(MESH)[5]
    with pytest.raises(native.NdsError) as e:
        native.HybridAmg(MESH, _rau(nvel), pressure_solver=1, **bad)
    assert e.value.code == -1  # NDS_E_INVALID
