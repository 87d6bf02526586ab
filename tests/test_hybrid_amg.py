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


# V-cycle cases: (hierarchy case, product options, oracle options); the
# reference's own device V-cycle results are in hybrid_amg_vcycle_r2.npz
VCYCLES = {
    "cheb2": ("exti_t60", {}, {}),
    "cheb2_deg3_aggr": ("direct_aggr_t40", dict(amg_cheb_degree=3), dict(cheb_degree=3)),
    "jacobi_2sweeps": ("exti_t60", dict(amg_smoother=1, amg_jacobi_fine_sweeps=2, amg_jacobi_coarse_sweeps=2,
                                        amg_jacobi_omega=0.6),
                       dict(smoother="jacobi", jacobi_fine_sweeps=2, jacobi_coarse_sweeps=2, jacobi_omega=0.6)),
    "l1jacobi": ("exti_t60", dict(amg_smoother=2), dict(smoother="l1jacobi")),
    "mcgs": ("exti_t60", dict(amg_smoother=3, amg_mcgs_omega=0.9), dict(smoother="mcgs", mcgs_omega=0.9)),
}
VGOLD = GOLDEN / "hybrid_amg_vcycle_r2.npz"


def _hierarchy(case):
    z = np.load(GOLD)
    arr = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(case + "/")}
    for k in z.files:
        if k.startswith("exti_t60/fine."):
            arr.setdefault(k.split("/", 1)[1], z[k])
    return arr


def _rel(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


@pytest.mark.parametrize("name", sorted(VCYCLES))
def test_vcycle_oracle_matches_reference_vcycle(name):
    """The oracle's V-cycle on the reference's hierarchy reproduces the
    reference's device V-cycle (its restriction sums with atomics: 1e-12)."""
    from oracle.hybrid_amg import VCycle
    case, _, oo = VCYCLES[name]
    v = np.load(VGOLD)
    z = VCycle(_hierarchy(case), oo).apply(v["b"])
    assert _rel(z, v[name]) < 1e-12, (name, _rel(z, v[name]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(VCYCLES))
def test_device_vcycle_matches_reference_vcycle(native, name):
    case, po, _ = VCYCLES[name]
    v = np.load(VGOLD)
    nvel = native.hybrid_counts(MESH)[5]
    z = native.hybrid_amg_vcycle(MESH, _rau(nvel), v["b"], pressure_solver=1, **CASES[case], **po)
    assert _rel(z, v[name]) < 1e-12, (name, _rel(z, v[name]))


def test_separate_post_vcycle_is_symmetric():
    """With its own post-smoothing work vectors the cheb2 V-cycle is a
    symmetric operator (x.My = y.Mx); the reference's, whose post-smoothing
    aliases the result and the Chebyshev product, is not."""
    from oracle.hybrid_amg import VCycle
    arr = _hierarchy("exti_t60")
    pin = int(arr["pin"][0])
    rng = np.random.default_rng(5)
    x, y = rng.standard_normal((2, len(arr["fine.diag"])))
    x[pin] = y[pin] = 0.0

    def gap(opt):
        V = VCycle(arr, opt)
        My, Mx = V.apply(y), V.apply(x)
        return abs(x @ My - y @ Mx) / (np.linalg.norm(x) * np.linalg.norm(My))

    assert gap(dict(separate_post=True)) < 1e-13
    assert gap({}) > 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cheb2", "jacobi_2sweeps"])
def test_device_separate_post_vcycle_matches_oracle(native, name):
    from oracle.hybrid_amg import VCycle
    case, po, oo = VCYCLES[name]
    v = np.load(VGOLD)
    nvel = native.hybrid_counts(MESH)[5]
    z = native.hybrid_amg_vcycle(MESH, _rau(nvel), v["b"], pressure_solver=1, amg_separate_post=1, **CASES[case],
                                 **po)
    want = VCycle(_hierarchy(case), dict(oo, separate_post=True)).apply(v["b"])
    assert _rel(z, want) < 1e-12, (name, _rel(z, want))


@pytest.mark.parametrize("args, message", [
    (["--bogus", "1"], "unknown argument --bogus"),
    (["--pressure-solver", "pcg_gmres"], "pressure solver must be pcg_amg or pcg_jacobi"),
    (["--amg-hierarchy", "sa"], "--amg-hierarchy must be cf"),
    (["--amg-smoother", "ilu"], "unknown AMG smoother"),
    (["--cf-interp", "classical"], "CF interp must be direct or exti"),
    (["--momentum-work", "sgs2"], "momentum-work must be fgs1, altgs1, or sgs1"),
    (["--alpha-u", "1.5"], "bad relaxation"),
    (["--p-max"], "missing value for --p-max"),
])
def test_hxt4b_executable_rejects_bad_flags(native, args, message):
    """Flag errors end the run before any device work, with exit code 2 and
    the reference's HXT4B_ERROR / HXT4B_GATE_STATUS=FAIL lines on stderr
    (hybrid_hxt4b/hxt4b_main.cu:218, 269)."""
    import subprocess
    from conftest import ROOT
    exe = ROOT / "nodals_b200" / "_lib" / "nodals_hxt4b_fp64"
    r = subprocess.run([str(exe), "--mesh", str(MESH), *args], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
    assert message in r.stderr and "HXT4B_GATE_STATUS=FAIL" in r.stderr


def test_flow_rejects_bad_pressure_options_before_device_work(native):
    """nds_hybrid_flow_fields checks its options before it looks for a
    device, so a bad preconditioner option is NDS_E_INVALID on any host."""
    import ctypes as C
    o = native.HybridFlowOptions.make(pressure_solver=1, amg_smoother=3, amg_mcgs_order=2)
    r = native.HybridFlowReport()
    rc = native.lib().nds_hybrid_flow_fields(str(MESH).encode(), C.byref(o), 0, 0, C.byref(r), None, None, None, None)
    assert rc == -1, native.lib().nds_last_error()
    assert b"symmetric MCGS" in native.lib().nds_last_error()
    o2 = native.HybridFlowOptions.make(pressure_solver=7)
    assert native.lib().nds_hybrid_flow_fields(str(MESH).encode(), C.byref(o2), 0, 0, C.byref(r), None, None, None,
                                               None) == -1
