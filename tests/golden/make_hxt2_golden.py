"""Golden log of the reference's HXT2 operator gate.

Runs the reference binary built from gpu/serial_cuda/hybrid_hxt2/hxt2_main.cu by
``make -C oracle ref`` (``oracle/_ref/nodals_hxt2_gpu``) on
``tests/golden/hxt1_hybrid_r2.bin`` with its defaults (nu 1, gamma 20) and
keeps its stdout as ``hxt2_hybrid_r2.log``.  Needs a CUDA device.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]

if __name__ == "__main__":
    r = subprocess.run([str(ROOT / "oracle" / "_ref" / "nodals_hxt2_gpu"), "--mesh", str(HERE / "hxt1_hybrid_r2.bin")],
                       capture_output=True, text=True, check=True)
    (HERE / "hxt2_hybrid_r2.log").write_text(r.stdout)
    print(r.stdout.splitlines()[-1])
