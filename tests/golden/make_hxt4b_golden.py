"""Golden logs of the reference's HXT4B mixed-mesh pipe SIMPLE.

Runs the reference binary built from gpu/serial_cuda/hybrid_hxt4b/hxt4b_main.cu
by ``make -C oracle ref`` (``oracle/_ref/nodals_hxt4b_fp64``) on
``tests/golden/hxt1_hybrid_r2.bin`` twice: with tight pressure solves
(``--p-rtol 1e-10 --p-max 2000``, kept as ``hxt4b_hybrid_r2_tight.log``) and
with its default controls except ``--p-max 400`` (the default 50 is too few
pressure iterations for this mesh in the first SIMPLE iteration; kept as
``hxt4b_hybrid_r2.log``).  The tight run's --vtu file is kept gzipped as
``hxt4b_hybrid_r2_tight.vtu.gz``.  Needs a CUDA device.
"""
from __future__ import annotations

import gzip
import subprocess
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
RUNS = {"hxt4b_hybrid_r2_tight.log": ["--p-rtol", "1e-10", "--p-max", "2000"], "hxt4b_hybrid_r2.log": ["--p-max", "400"]}

if __name__ == "__main__":
    with tempfile.TemporaryDirectory() as tmp:
        for name, extra in RUNS.items():
            vtu = Path(tmp) / (name + ".vtu")
            r = subprocess.run([str(ROOT / "oracle" / "_ref" / "nodals_hxt4b_fp64"), "--mesh",
                                str(HERE / "hxt1_hybrid_r2.bin"), "--vtu", str(vtu), *extra],
                               capture_output=True, text=True, check=True)
            (HERE / name).write_text(r.stdout.replace(str(vtu), "/dev/null"))
            if "tight" in name:
                (HERE / "hxt4b_hybrid_r2_tight.vtu.gz").write_bytes(gzip.compress(vtu.read_bytes(), mtime=0))
            print(name, r.stdout.splitlines()[-1])
