"""Golden setup of the mixed-mesh pressure preconditioner, from the reference's
own builders.

Runs ``oracle/_ref/ref_hybrid_amg_dump`` (built by ``make -C oracle ref`` from
the reference's hybrid_hxt4b/hxt4b_main.cu and hybrid_hxt5b/hybrid_amg.cuh,
hybrid_cf_overload.inc) on ``tests/golden/hxt1_hybrid_r2.bin`` with the rAU
vector ``rau(g) = 0.02 (1.5 + sin(0.37 (g + 1)))`` and keeps, per case, the
pressure matrix (first case only) and the CF hierarchy as
``hybrid_amg_r2.npz`` (keys ``<case>/<array>``).  Runs on the CPU; needs
the reference tree only through the built harness.

With ``--vcycle`` (needs a CUDA device) it also applies the reference's device
preconditioner once, for each smoother case of ``VCYCLES``, to the seeded
vector ``b`` (standard normal from seed 11, zero at the pin) and keeps ``b``
and each ``z = M^-1 b`` as ``hybrid_amg_vcycle_r2.npz``.
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

from oracle.dump import read_dump  # noqa: E402

MESH = HERE / "hxt1_hybrid_r2.bin"
# case -> harness flags (the product's options of the same meaning are set by the test)
CASES = {
    "exti_t60": ["--amg-terminal", "60"],
    "direct_aggr_t40": ["--amg-terminal", "40", "--cf-interp", "direct", "--cf-aggressive-first", "1",
                        "--cf-pmax", "4", "--cf-theta", "0.3"],
}


# V-cycle case -> (hierarchy case, harness smoother flags)
VCYCLES = {
    "cheb2": ("exti_t60", ["--amg-smoother", "cheb2"]),
    "cheb2_deg3_aggr": ("direct_aggr_t40", ["--amg-smoother", "cheb2", "--amg-cheb-degree", "3"]),
    "jacobi_2sweeps": ("exti_t60", ["--amg-smoother", "jacobi", "--amg-jacobi-fine-sweeps", "2",
                                    "--amg-jacobi-coarse-sweeps", "2", "--amg-jacobi-omega", "0.6"]),
    "l1jacobi": ("exti_t60", ["--amg-smoother", "l1jacobi"]),
    "mcgs": ("exti_t60", ["--amg-smoother", "mcgs", "--amg-mcgs-omega", "0.9"]),
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
    if "--vcycle" in sys.argv[1:]:
        vcycles(nvel)


def vcycles(nvel: int) -> None:
    z = np.load(HERE / "hybrid_amg_r2.npz")
    pin = int(z["exti_t60/pin"][0])
    npres = len(z["exti_t60/fine.diag"])
    b = np.random.default_rng(11).standard_normal(npres)
    b[pin] = 0.0
    out = {"b": b}
    with tempfile.TemporaryDirectory() as td:
        rp, bp = Path(td) / "rau.bin", Path(td) / "b.bin"
        rau_of(nvel).astype("<f8").tofile(rp)
        b.astype("<f8").tofile(bp)
        for name, (case, flags) in VCYCLES.items():
            zp = Path(td) / f"{name}.z"
            subprocess.run([str(ROOT / "oracle" / "_ref" / "ref_hybrid_amg_dump"), "--mesh", str(MESH), "--rau", str(rp),
                            "--out", str(Path(td) / "dump.bin"), *CASES[case], *flags, "--apply", str(bp),
                            "--z-out", str(zp)], check=True, stdout=subprocess.DEVNULL)
            out[name] = np.fromfile(zp, dtype="<f8")
    np.savez_compressed(HERE / "hybrid_amg_vcycle_r2.npz", **out)


if __name__ == "__main__":
    main()
