"""Golden log of the reference's HXT3A divergence gate.

Runs the reference binary built from gpu/serial_cuda/hybrid_hxt3a/hxt3a_main.cu
by ``make -C oracle ref`` (``oracle/_ref/nodals_hxt3a_gpu``) on
``tests/golden/hxt1_hybrid_r2.bin`` and keeps its stdout as
``hxt3a_hybrid_r2.log`` (its exit code too: 3 when one of the gate's own
checks fails, which still prints every line).  Needs a CUDA device.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]

if __name__ == "__main__":
    r = subprocess.run([str(ROOT / "oracle" / "_ref" / "nodals_hxt3a_gpu"), "--mesh", str(HERE / "hxt1_hybrid_r2.bin")],
                       capture_output=True, text=True)
    if r.returncode not in (0, 3):
        raise SystemExit(r.stderr)
    (HERE / "hxt3a_hybrid_r2.log").write_text(r.stdout + f"EXIT_CODE={r.returncode}\n")
    print(r.stdout.splitlines()[-1])
