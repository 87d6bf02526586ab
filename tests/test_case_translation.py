"""The .case front end maps keys onto the drop-in CLI exactly as the reference
launcher does (reference tests: tests/test_gpu_case_translation.py,
tests/test_gpu_supg_case_translation.py)."""
from __future__ import annotations

import subprocess
import sys

import pytest

from conftest import ROOT
from nodals_b200 import case as mod

CASE = mod.DEFAULT_CASE


def pairs(opts):
    assert len(opts) % 2 == 0, opts
    return {opts[i]: opts[i + 1] for i in range(0, len(opts), 2)}


def test_canonical_case_selects_cf_pmis_family():
    cp = mod.Case.read(CASE)
    o = pairs(mod.command_line(cp))
    assert o["--amg-hierarchy"] == "cf"
    assert o["--cf-coarsening"] == "pmis"
    assert o["--cf-strength"] == "classical-negative"
    assert o["--cf-theta"] == "0.25"
    assert o["--cf-interp"] == "exti"
    assert o["--cf-pmax"] == "8"
    assert o["--cf-aggressive-first"] == "0"
    assert o["--amg-smoother"] == "jacobi"
    assert o["--pressure-solver"] == "richardson"
    assert o["--pressure-richardson-omega"] == "1.0"
    assert o["--fine-csr-refresh-every"] == "1"
    assert o["--momentum-work"] == "fgs1"
    assert o["--run-mode"] == "converge"
    assert mod.precision_of(cp) == "fp32"


def test_sa_cheb_pcg_is_three_keys_away():
    cp = mod.Case.read(CASE)
    cp.set("pressure_amg", "hierarchy", "sa")
    cp.set("pressure_amg", "smoother", "cheb2")
    cp.set("pressure", "solver", "pcg")
    o = pairs(mod.command_line(cp))
    assert o["--amg-hierarchy"] == "sa"
    assert o["--amg-smoother"] == "cheb2"
    assert o["--amg-spectrum-policy"] == "auto"
    assert o["--amg-power-its"] == "16"
    assert o["--amg-cheb-degree"] == "2"
    assert o["--pressure-solver"] == "pcg"


def test_l1jacobi_and_outer_chebyshev():
    cp = mod.Case.read(CASE)
    cp.set("pressure_amg", "smoother", "l1jacobi")
    cp.set("pressure", "solver", "cheb")
    o = pairs(mod.command_line(cp))
    assert o["--amg-smoother"] == "l1jacobi"
    assert o["--pressure-solver"] == "cheb"
    assert o["--pressure-cheb-degree"] == "3"
    assert o["--pressure-power-its"] == "6"


def test_fixed10_consistency():
    cp = mod.Case.read(CASE)
    cp.set("run", "run_mode", "fixed10")
    cp.set("simple", "max_iterations", "10")
    o = pairs(mod.command_line(cp))
    assert o["--run-mode"] == "fixed10"
    assert o["--max-outer"] == "10"
    cp.set("simple", "max_iterations", "11")
    with pytest.raises(ValueError, match="requires"):
        mod.command_line(cp)


def test_cheb2_without_spectrum_rejected():
    cp = mod.Case.read(CASE)
    cp.set("pressure_amg", "smoother", "cheb2")
    cp.set("pressure_amg", "spectrum_policy", "off")
    with pytest.raises(ValueError, match="requires spectrum_policy"):
        mod.command_line(cp)


def test_unknown_key_rejected():
    cp = mod.Case.read(CASE)
    with pytest.raises(ValueError, match="unknown GPU case key"):
        cp.set("pressure_amg", "smother", "jacobi")
    cp.values[("pressure_amg", "smother")] = "jacobi"
    with pytest.raises(ValueError, match="unknown GPU case key"):
        mod.command_line(cp)


def test_set_override_and_unknown_section():
    cp = mod.Case.read(CASE)
    cp.override(["pressure.rtol=1e-4", "simple.alpha_u=0.7"])
    o = pairs(mod.command_line(cp))
    assert o["--p-rtol"] == "1e-4" and o["--alpha-u"] == "0.7"
    with pytest.raises(ValueError, match="unknown GPU case section"):
        cp.override(["bogus.x=1"])


def test_supg_translation_and_rejections():
    cp = mod.Case.read(CASE)
    for k, v in (("enabled", "true"), ("tau_scale", "0.05"), ("magic", "9.0"), ("form", "implicit"), ("quad_points", "64")):
        cp.set("supg", k, v)
    o = pairs(mod.command_line(cp))
    assert o["--supg"] == "1" and o["--supg-quad-points"] == "64" and o["--supg-form"] == "implicit"
    cp.set("supg", "enabled", "false")
    assert pairs(mod.command_line(cp))["--supg"] == "0"
    cp.set("supg", "enabled", "true")
    cp.set("supg", "form", "explicit")
    with pytest.raises(ValueError, match="form=implicit"):
        mod.command_line(cp)
    cp.set("supg", "form", "implicit")
    cp.set("supg", "quad_points", "27")
    with pytest.raises(ValueError, match="quad_points=64"):
        mod.command_line(cp)


def test_dry_run_and_missing_solver(tmp_path, monkeypatch):
    r = subprocess.run([sys.executable, "-m", "nodals_b200.case", str(CASE), "--dry-run", "--dump-options-json"],
                       capture_output=True, text=True, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert "NODALS_GPU_CASE_RESULT status=DRY_RUN" in r.stdout
    assert "NODALS_GPU_OPTIONS_JSON=" in r.stdout
    monkeypatch.setattr(mod, "PACKAGE_LIB", tmp_path)
    monkeypatch.delenv("NODALS_GPU_FP32_EXE", raising=False)
    assert mod.main([str(CASE), "--exe", str(tmp_path / "none"), "--set", f"run.output_root={tmp_path}"]) == 2
    bad = tmp_path / "bad.case"
    bad.write_text("[run]\nnonsense = 1\n")
    r = subprocess.run([sys.executable, "-m", "nodals_b200.case", str(bad), "--dry-run"], capture_output=True,
                       text=True, cwd=ROOT)
    assert r.returncode == 4 and "unknown GPU case key" in r.stderr


def test_messages_and_defaults_from_the_key_table():
    """Defaults of the reference's case schema and its error wording."""
    cp = mod.Case.read(CASE)
    for k in [k for k in list(cp.values) if k[0] != "solver"]:
        del cp.values[k]
    o = pairs(mod.command_line(cp))
    assert o["--tag"] == "nodals_gpu" and o["--simple-tol"] == "1e-3" and o["--max-outer"] == "2500"
    assert o["--amg-hierarchy"] == "cf" and o["--amg-smoother"] == "jacobi"
    assert o["--pressure-solver"] == "richardson" and o["--p-rtol"] == "0.5" and o["--p-max"] == "20"
    assert o["--wall"] == "patch_0_0" and o["--inlet"] == "patch_2_0" and o["--outlet"] == "patch_1_0"
    assert mod.precision_of(cp) == "fp32"
    cases = [(("pressure", "solver", "gmres"), "[pressure] solver must be pcg, richardson, or cheb"),
             (("pressure_amg", "hierarchy", "rs"), "[pressure_amg] hierarchy must be sa or cf"),
             (("run", "precision", "fp16"), "[run] precision must be fp32 or fp64"),
             (("momentum", "work", "sgs1"), "current H8 supports only [momentum] work=fgs1"),
             (("pressure_amg_cf", "coarsening", "hmis"),
              "current H8 CF hierarchy supports only [pressure_amg_cf] coarsening=pmis"),
             (("pressure", "fine_csr_refresh_every", "2"), "current H8 requires [pressure] fine_csr_refresh_every=1"),
             (("supg", "enabled", "maybe"), "[supg] enabled: expected boolean, got 'maybe'")]
    for (sec, key, val), msg in cases:
        c = mod.Case.read(CASE)
        c.set(sec, key, val)
        with pytest.raises(ValueError) as e:
            mod.command_line(c)
        assert str(e.value) == msg
    c = mod.Case.read(CASE)
    del c.values[("solver", "mesh")]
    with pytest.raises(ValueError, match=r"missing required \[solver\] mesh"):
        mod.command_line(c)
