"""Golden log of the reference's HXT4A mixed hex/tet Stokes gate.

Runs the reference binary built from gpu/serial_cuda/hybrid_hxt4a/hxt4a_main.cu
by ``make -C oracle ref`` (``oracle/_ref/nodals_hxt4a_fp64``) with its
default controls on ``tests/golden/hxt1_hybrid_r2.bin`` (made by
make_hxt1_golden.py) and keeps its stdout as
``tests/golden/hxt4a_hybrid_r2.log``.  Needs a CUDA device.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]

if __name__ == "__main__":
    out = subprocess.run([str(ROOT / "oracle" / "_ref" / "nodals_hxt4a_fp64"), "--mesh", str(HERE / "hxt1_hybrid_r2.bin")],
                         capture_output=True, text=True, check=True).stdout
    (HERE / "hxt4a_hybrid_r2.log").write_text(out)
    print(out.splitlines()[-1])
