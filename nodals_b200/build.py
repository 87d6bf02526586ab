"""In-tree build of the native library and the drop-in executables.

Outputs (git-ignored, shipped with the working tree):
  nodals_b200/_lib/libnodals_b200.so      C ABI (include/nodals_b200.h)
  nodals_b200/_lib/nodals_gpu_h8_fp64     drop-in for the reference's nodals_gpu_h8_fp64
  nodals_b200/_lib/nodals_gpu_h8_fp32     drop-in for the reference's nodals_gpu_h8_fp32

Every CUDA source is compiled for sm_100a only.  Incremental: an object is
rebuilt when its source or any header of the package is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "_lib"
NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("NDS_CXX", "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wextra", "-Wno-unused-parameter", "-ffp-contract=off"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fopenmp",
           "-Xptxas", "-O3"] + ARCH


def _headers():
    return [p for p in list(CSRC.rglob("*.hpp")) + list(CSRC.rglob("*.cuh")) + [ROOT / "include" / "nodals_b200.h"]]


def _stale(obj: Path, src: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    newest = max(p.stat().st_mtime for p in _headers())
    lib_srcs = sorted((CSRC / "host").glob("*.cpp")) + [CSRC / "capi_host.cpp"]
    cu_srcs = sorted((CSRC / "cuda").glob("*.cu")) if (CSRC / "cuda").exists() else []
    jobs_ = []
    objs = []
    for s in lib_srcs:
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if _stale(o, s, newest):
            jobs_.append([CXX, *CXXFLAGS, "-I", str(CSRC), "-c", str(s), "-o", str(o)])
    for s in cu_srcs:
        o = BUILD / (s.stem + ".cu.o")
        objs.append(o)
        if _stale(o, s, newest):
            # the mixed-mesh solvers capture their default-stream launches into graphs
            extra = ["--default-stream", "per-thread"] if s.name == "hybrid.cu" else []
            jobs_.append([NVCC, *NVFLAGS, *extra, "-I", str(CSRC), "-c", str(s), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for out in ex.map(_run, jobs_):
            if verbose and out.strip():
                print(out)
    so = LIB / "libnodals_b200.so"
    if not so.exists() or any(o.stat().st_mtime > so.stat().st_mtime for o in objs):
        _run([NVCC, "-shared", *ARCH, "-o", str(so), *map(str, objs), "-Xcompiler", "-fopenmp", "-lcudart"])
    cli = CSRC / "cli" / "nodals_gpu_h8.cpp"
    if cli.exists():
        exe = LIB / "nodals_gpu_h8_fp64"
        if not exe.exists() or exe.stat().st_mtime < max(cli.stat().st_mtime, so.stat().st_mtime, newest):
            _run([CXX, *CXXFLAGS, "-I", str(CSRC), "-o", str(exe), str(cli), "-L", str(LIB), "-lnodals_b200",
                  "-Wl,-rpath,$ORIGIN"])
            shutil.copy2(exe, LIB / "nodals_gpu_h8_fp32")
    for name in ("nodals_hxt4a", "nodals_hxt4b"):
        gate = CSRC / "cli" / f"{name}.cpp"
        exe = LIB / f"{name}_fp64"
        if gate.exists() and (not exe.exists() or exe.stat().st_mtime < max(gate.stat().st_mtime, so.stat().st_mtime, newest)):
            _run([CXX, *CXXFLAGS, "-I", str(CSRC), "-o", str(exe), str(gate), "-L", str(LIB), "-lnodals_b200",
                  "-Wl,-rpath,$ORIGIN"])
    return so


if __name__ == "__main__":
    p = build(verbose="-v" in sys.argv)
    print(p)
