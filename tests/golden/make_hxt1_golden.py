"""Golden HXT1 file made by the reference's own converter.

Writes the seeded ``pipe_tiny`` mesh as MSH 2.2 with this package's writer,
converts it with the reference's ``turbulence/sst_gpu_v2/tools/msh2_to_hxt1.py``
(which runs its ``prepare_hxt1.py``) and keeps the resulting
``HXT1_mesh.bin`` as ``tests/golden/hxt1_pipe_tiny.bin``; writes the small
mixed hex/tet pipe ``HYBRID`` as HXT0 arrays and keeps the reference
preparer's ``HXT1_mesh.bin`` of it as ``tests/golden/hxt1_hybrid_r2.bin``.  Needs the
reference tree (first argument, default: oracle.refpath.reference_root()); the
tests only read the committed file.
"""
from __future__ import annotations

import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from nodals_b200 import meshgen  # noqa: E402
from oracle.refpath import reference_root  # noqa: E402


# the small mixed pipe: 2 hex rings, 8 sectors, 20 slabs, R = 0.5, L = 10 (10 D)
HYBRID = dict(nr=2, ntheta=8, nz=20, radius=0.5, length=10.0)


def main() -> None:
    ref = Path(sys.argv[1]) if len(sys.argv) > 1 else reference_root()
    if ref is None:
        raise SystemExit("reference tree not found: pass its path or set NODALS_REFERENCE")
    conv = ref / "turbulence" / "sst_gpu_v2" / "tools" / "msh2_to_hxt1.py"
    with tempfile.TemporaryDirectory() as tmp:
        msh = meshgen.write_msh2(meshgen.named("pipe_tiny"), Path(tmp) / "pipe_tiny.msh")
        subprocess.run([sys.executable, str(conv), "--msh", str(msh), "--out", str(Path(tmp) / "out")], check=True,
                       stdout=subprocess.DEVNULL)
        shutil.copy(Path(tmp) / "out" / "HXT1_mesh.bin", HERE / "hxt1_pipe_tiny.bin")
        # mixed hex/tet pipe through the reference's HXT1 preparer
        hx = meshgen.write_hxt0(meshgen.hybrid_pipe(**HYBRID), Path(tmp) / "hxt0.npz")
        prep = ref / "gpu" / "serial_cuda" / "hybrid_hxt1" / "prepare_hxt1.py"
        subprocess.run([sys.executable, str(prep), "--input", str(hx), "--outdir", str(Path(tmp) / "hyb")], check=True,
                       stdout=subprocess.DEVNULL)
        shutil.copy(Path(tmp) / "hyb" / "HXT1_mesh.bin", HERE / "hxt1_hybrid_r2.bin")
    print("wrote", HERE / "hxt1_pipe_tiny.bin", HERE / "hxt1_hybrid_r2.bin")


if __name__ == "__main__":
    main()
