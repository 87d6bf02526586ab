"""Golden setup of the mixed-mesh pressure preconditioner, from the reference's
own builders.

Runs ``oracle/_ref/ref_hybrid_amg_dump`` (built by ``make -C oracle ref`` from
the reference's hybrid_hxt4b/hxt4b_main.cu and hybrid_hxt5b/hybrid_amg.cuh,
hybrid_cf_overload.inc) on ``tests/golden/hxt1_hybrid_r2.bin`` with the rAU
vector ``rau(g) = 0.02 (1.5 + sin(0.37 (g + 1)))`` and keeps, per case, the
pressure matrix (first case only) and the CF hierarchy as
``hybrid_amg_r2.npz`` (keys ``<case>/<array>``).  Runs on the CPU; needs
the reference tree only through the built harness.
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from nodals_b200.native import read_dump  # noqa: E402

MESH = HERE / "hxt1_hybrid_r2.bin"
# case -> harness flags (the product's options of the same meaning are set by the test)
CASES = {
    "exti_t60": ["--amg-terminal", "60"],
    "direct_aggr_t40": ["--amg-terminal", "40", "--cf-interp", "direct", "--cf-aggressive-first", "1",
                        "--cf-pmax", "4", "--cf-theta", "0.3"],
}


def rau_of(nvel: int) -> np.ndarray:
    g = np.arange(nvel, dtype=np.float64)
    return 0.02 * (1.5 + np.sin(0.37 * (g + 1)))


def main() -> None:
    from oracle.hybrid_vtu import read_mixed_hxt1
    nvel = int(read_mixed_hxt1(MESH)["counts"][5])
    out = {}
    with tempfile.TemporaryDirectory() as td:
        rp = Path(td) / "rau.bin"
        rau_of(nvel).astype("<f8").tofile(rp)
        for case, flags in CASES.items():
            dump = Path(td) / f"{case}.bin"
            subprocess.run([str(ROOT / "oracle" / "_ref" / "ref_hybrid_amg_dump"), "--mesh", str(MESH), "--rau", str(rp),
                            "--out", str(dump), *flags], check=True, stdout=subprocess.DEVNULL)
            for k, v in read_dump(dump).items():
                # the pressure matrix depends on rAU only: kept once
                if not k.startswith("b.") and (case == "exti_t60" or not k.startswith("fine.")):
                    out[f"{case}/{k}"] = v
    np.savez_compressed(HERE / "hybrid_amg_r2.npz", **out)


if __name__ == "__main__":
    main()
