"""The C ABI: every function declared in include/nodals_b200.h is exported
by the built library, and a plain C program can drive the host side of it.
On a machine without a CUDA device the solver must refuse to start
(NDS_E_CUDA) rather than fall back to anything."""
from __future__ import annotations

import ctypes
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "nodals_b200.h"
LIBDIR = ROOT / "nodals_b200" / "_lib"


def declared_functions() -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(nds_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported(native):
    lib = ctypes.CDLL(str(LIBDIR / "libnodals_b200.so"))
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_c_program_drives_host_abi(native, meshes, tmp_path):
    from nodals_b200 import meshgen
    msh = tmp_path / "tiny.msh"
    meshgen.write_msh2(meshes("pipe_tiny"), str(msh))
    exe = tmp_path / "abi_smoke"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", f"-I{ROOT / 'include'}", str(ROOT / "tests/c/abi_smoke.c"),
                    f"-L{LIBDIR}", "-lnodals_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), str(msh)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = dict(l.split(" ", 1) for l in out.stdout.strip().splitlines())
    assert lines["mesh"].split()[1] == "720"
    st = int(lines["solver_create"].split()[0])
    import torch
    if torch.cuda.is_available():
        assert st == 0
    else:
        assert st == -3, lines["solver_create"]
