"""Binary HXT1 meshes (the reference's hybrid/SST mesh format,
gpu/serial_cuda/hybrid_hxt1/hxt1_mesh.hpp:19-103).

* The C++ reader, given the file the reference's own converter
  (turbulence/sst_gpu_v2/tools/msh2_to_hxt1.py) made from the seeded
  pipe_tiny mesh, yields bit for bit the setup of the MSH 2.2 reader on the
  same mesh.
* The Python writer reproduces that file: every count, index and record
  identical, points identical, geometry within 1e-13 relative (the
  reference takes det and J^-1 from LU factorisations, the writer from
  cofactors).
* Malformed files are rejected with the reference loader's checks (magic,
  version, short read, trailing bytes), and files with hex cells are
  refused.
"""
from __future__ import annotations

import struct

import numpy as np
import pytest

from conftest import GOLDEN

GOLD = GOLDEN / "hxt1_pipe_tiny.bin"
ARRAYS = ["mesh.tets", "mesh.opp_face", "mesh.face_patch", "mesh.xyz", "mom.row", "mom.col", "mom.val",
          "color.offset", "color.rows", "cell.ref", "cell.bcoeff", "fine.row", "fine.col", "fine.slot"]
OPTS = dict(max_outer=10, amg_terminal=60)


def _parse(path):
    b = open(path, "rb").read()
    assert b[:8] == b"HXT1BIN1"
    h = struct.unpack_from("<II13Q", b, 8)
    nv, nhex, nt, _, ntf, nvel, npr, nif, nwh, nih, nit, noh, not_ = h[2:]
    off = 8 + 8 + 8 * 13
    out = {"header": h}
    for name, n, dt, w in (("points", nv, "<f8", 3), ("tets", nt, "<i4", 4), ("tvel", nt, "<i4", 8),
                           ("tp", nt, "<i4", 1), ("geom", nt, "<f8", 12), ("in", nit, "<i4", 3),
                           ("out", not_, "<i4", 3)):
        a = np.frombuffer(b, dtype=dt, count=n * w, offset=off).reshape(n, w)
        off += a.nbytes
        out[name] = a
    assert off == len(b)
    return out


def test_reader_matches_msh2_setup(native, meshes, tmp_path):
    from nodals_b200 import meshgen
    msh = meshgen.write_msh2(meshes("pipe_tiny"), tmp_path / "m.msh")
    Pm = native.Problem(native.Mesh.read_msh2(msh), **OPTS)
    Ph = native.Problem(native.Mesh.read_hxt1(GOLD), **OPTS)
    assert Pm.counts() == Ph.counts()
    for name in ARRAYS:
        assert np.array_equal(Pm.array(name), Ph.array(name)), name


def test_writer_matches_reference_converter(meshes, tmp_path):
    from nodals_b200 import meshgen
    ours = _parse(meshgen.write_hxt1(meshes("pipe_tiny"), tmp_path / "m.bin"))
    ref = _parse(GOLD)
    assert ours["header"] == ref["header"]
    for k in ("points", "tets", "tvel", "tp", "in", "out"):
        assert np.array_equal(ours[k], ref[k]), k
    g, r = ours["geom"], ref["geom"]
    assert np.all(np.abs(g - r) <= 1e-13 * np.maximum(np.abs(r), np.abs(r).max(axis=0)))


def _bad(tmp_path, data, name):
    p = tmp_path / name
    p.write_bytes(data)
    return p


@pytest.mark.parametrize("case,message", [
    ("magic", "bad HXT1 magic"), ("version", "unsupported HXT1 version"), ("short", "short read"),
    ("trailing", "trailing bytes"), ("hex", "pure-tet HXT1"),
])
def test_reader_rejects(native, tmp_path, case, message):
    b = bytearray(GOLD.read_bytes())
    if case == "magic":
        b[:8] = b"HXT0BIN1"
    elif case == "version":
        b[8:12] = struct.pack("<I", 2)
    elif case == "short":
        b = b[:-5]
    elif case == "trailing":
        b += b"\0"
    elif case == "hex":
        b[16 + 8:16 + 16] = struct.pack("<Q", 1)  # nhex
    with pytest.raises(native.NdsError) as e:
        native.Mesh.read_hxt1(_bad(tmp_path, bytes(b), case + ".bin"))
    assert e.value.code == -2 and message in str(e.value)


def test_hybrid_writer_matches_reference_preparer(tmp_path):
    """meshgen.write_hxt1_hybrid against the reference preparer's file of the
    same mixed pipe (tests/golden/hxt1_hybrid_r2.bin, made by
    make_hxt1_golden.py): every count, index and record identical, points and
    geometry to 1e-13 of each record's largest entry (here the files are
    byte-identical; the reference takes det J and J^-1 from LAPACK through
    numpy, so a different LAPACK build may move the last bit)."""
    import sys
    from oracle.hybrid_vtu import read_mixed_hxt1
    from nodals_b200 import meshgen
    sys.path.insert(0, str(GOLDEN))
    from make_hxt1_golden import HYBRID
    p = meshgen.write_hxt1_hybrid(meshgen.hybrid_pipe(**HYBRID), tmp_path / "r2.bin")
    got, want = read_mixed_hxt1(p), read_mixed_hxt1(GOLDEN / "hxt1_hybrid_r2.bin")
    assert got["counts"] == want["counts"]
    for k, w in want.items():
        if k == "counts":
            continue
        g = got[k]
        assert g.shape == w.shape, k
        if w.dtype.kind == "f":
            scale = np.maximum(np.abs(w).max(axis=1, keepdims=True), 1e-300) if w.size else 1.0
            assert np.all(np.abs(g - w) <= 1e-13 * scale), k
        else:
            assert np.array_equal(g, w), k


def test_hybrid_writer_rejects_bad_records(tmp_path):
    from nodals_b200 import meshgen
    m = meshgen.hybrid_pipe(nr=2, ntheta=8, nz=4, radius=0.5, length=2.0)
    # the top face of a hex in the first slab is shared with the next slab's hex
    m.wall_quads = np.concatenate((m.wall_quads, m.hexes[:1, 4:8]))
    with pytest.raises(ValueError, match="owner count"):
        meshgen.write_hxt1_hybrid(m, tmp_path / "bad.bin")
