"""The 64-point collapsed rule of the SUPG terms (exported as supg.rule).

Checked against scipy's Gauss-Jacobi roots (an independent computation) and,
when the reference tree is present, against the node/weight table of the
reference's host SUPG twin (gpu/serial_cuda/g4_host.hpp:330-335), to 1e-15.
"""
from __future__ import annotations

import re

import numpy as np
import pytest
from scipy.special import roots_jacobi

from conftest import REFERENCE


def _rule01(n, alpha):
    x, w = roots_jacobi(n, alpha, 0.0)
    # (1-x)^alpha dx on [-1,1] -> 2^(alpha+1) (1-r)^alpha dr on [0,1]
    return (x + 1) / 2, w / 2 ** (alpha + 1)


def _product_rule(nodes):
    (rn, rw), (sn, sw), (tn, tw) = nodes
    out = []
    for ir in range(4):
        for is_ in range(4):
            for it in range(4):
                r, s, t = rn[ir], sn[is_], tn[it]
                lam = [(1 - r) * (1 - s) * (1 - t), r, (1 - r) * s, (1 - r) * (1 - s) * t]
                out.append(lam + [rw[ir] * sw[is_] * tw[it]])
    return np.array(out)


def _problem(native, meshes):
    return native.Problem(native.Mesh.from_tetmesh(meshes("pipe_tiny")), max_outer=10, amg_terminal=60)


def test_supg_rule_matches_gauss_jacobi(native, meshes):
    rule = _problem(native, meshes).array("supg.rule").reshape(64, 5)
    want = _product_rule([_rule01(4, 2), _rule01(4, 1), _rule01(4, 0)])
    assert np.max(np.abs(rule - want)) <= 1e-15
    assert abs(rule[:, 4].sum() - 1.0 / 6.0) <= 1e-15


@pytest.mark.skipif(REFERENCE is None or not (REFERENCE / "gpu/serial_cuda/g4_host.hpp").exists(),
                    reason="reference tree absent")
def test_supg_rule_matches_reference_table(native, meshes):
    text = (REFERENCE / "gpu/serial_cuda/g4_host.hpp").read_text()
    i = text.index("host_add_supg64_g4")
    tab = {}
    for name in ("rn", "rw", "sn", "sw", "tn", "tw"):
        m = re.search(r"const double " + name + r"\[4\]=\{([^}]*)\}", text[i:])
        tab[name] = [float(v) for v in m.group(1).split(",")]
    want = _product_rule([(tab["rn"], tab["rw"]), (tab["sn"], tab["sw"]), (tab["tn"], tab["tw"])])
    rule = _problem(native, meshes).array("supg.rule").reshape(64, 5)
    assert np.max(np.abs(rule - want)) <= 1e-15
