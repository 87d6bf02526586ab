"""CPU restatement of the mixed-mesh VTU of the reference's HXT4B executable
-- test infrastructure.

``read_mixed_hxt1`` parses a binary HXT1 file with hex and tet cells in the
record order of gpu/serial_cuda/hybrid_hxt1/hxt1_mesh.hpp:19-103 (header,
points, hexes, tets, velocity dofs, pressure ids, geometry, interface and
boundary records).  ``vtu_text`` renders the file that
hybrid_hxt4b/hxt4b_main.cu:203-209 writes for ``--vtu``: 16 significant
digits, hexes (VTK 12) before tets (VTK 10), vertex pressure as the
volume-weighted average of the P0 cells around the vertex, each cell giving
V/8 (hex) or V/4 (tet), summed in extended precision in cell order.
"""
from __future__ import annotations

import struct

import numpy as np


def read_mixed_hxt1(path) -> dict:
    b = open(path, "rb").read()
    if b[:8] != b"HXT1BIN1":
        raise ValueError("bad HXT1 magic")
    version, _ = struct.unpack_from("<II", b, 8)
    if version != 1:
        raise ValueError("unsupported HXT1 version")
    n = struct.unpack_from("<13Q", b, 16)
    nv, nh, nt, _, _, nvel, npr, nif, nwh, nih, nit, noh, not_ = n
    off = 16 + 8 * 13
    out = {"counts": n}
    for name, cnt, dt, w in (("points", nv, "<f8", 3), ("hexes", nh, "<i4", 8), ("tets", nt, "<i4", 4),
                             ("hex_dofs", nh, "<i4", 14), ("tet_dofs", nt, "<i4", 8), ("hex_p", nh, "<i4", 1),
                             ("tet_p", nt, "<i4", 1), ("hex_geom", nh, "<f8", 82), ("tet_geom", nt, "<f8", 12),
                             ("interface", nif, "<i4", 9), ("wall_hex", nwh, "<i4", 3), ("in_hex", nih, "<i4", 3),
                             ("in_tet", nit, "<i4", 3), ("out_hex", noh, "<i4", 3), ("out_tet", not_, "<i4", 3)):
        a = np.frombuffer(b, dtype=dt, count=cnt * w, offset=off).reshape(cnt, w)
        off += a.nbytes
        out[name] = a
    if off != len(b):
        raise ValueError("trailing bytes in HXT1 file")
    return out


def _g(x) -> str:
    return "%.16g" % float(x)


def vertex_pressure(m: dict, p) -> np.ndarray:
    """Volume-weighted vertex average of the cell pressures (pure-Python loop
    in the reference's accumulation order; small meshes only)."""
    nv = int(m["counts"][0])
    nh = len(m["hexes"])
    w = [np.longdouble(0)] * nv
    pa = [np.longdouble(0)] * nv
    for cells, geom, k, base in ((m["hexes"], m["hex_geom"], 8, 0), (m["tets"], m["tet_geom"], 4, nh)):
        for c in range(len(cells)):
            share = float(geom[c, 0]) / k
            contrib = share * float(p[base + c])
            for v in cells[c]:
                w[v] += np.longdouble(share)
                pa[v] += np.longdouble(contrib)
    return np.array([float(pa[i] / w[i]) if w[i] > 0 else 0.0 for i in range(nv)])


def vtu_text(m: dict, u0, u1, u2, p) -> str:
    nv = int(m["counts"][0])
    nh, nt = len(m["hexes"]), len(m["tets"])
    out = ['<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">\n',
           f'<UnstructuredGrid><Piece NumberOfPoints="{nv}" NumberOfCells="{nh + nt}">\n',
           '<Points><DataArray type="Float64" NumberOfComponents="3" format="ascii">\n']
    out += [f"{_g(x)} {_g(y)} {_g(z)}\n" for x, y, z in m["points"]]
    out.append('</DataArray></Points><Cells><DataArray type="Int32" Name="connectivity" format="ascii">\n')
    out += ["".join(f"{int(v)} " for v in cell) + "\n" for cell in (*m["hexes"], *m["tets"])]
    out.append('</DataArray><DataArray type="Int64" Name="offsets" format="ascii">\n')
    ends = np.cumsum([8] * nh + [4] * nt)
    out += [f"{int(e)}\n" for e in ends]
    out.append('</DataArray><DataArray type="UInt8" Name="types" format="ascii">\n')
    out += ["12\n"] * nh + ["10\n"] * nt
    out.append('</DataArray></Cells><PointData><DataArray type="Float64" Name="velocity_Q1P1_vertex" '
               'NumberOfComponents="3" format="ascii">\n')
    out += [f"{_g(u0[i])} {_g(u1[i])} {_g(u2[i])}\n" for i in range(nv)]
    out.append('</DataArray><DataArray type="Float64" Name="pressure_Q0P0_vertex_volume_average" format="ascii">\n')
    out += [_g(x) + "\n" for x in vertex_pressure(m, p)]
    out.append('</DataArray></PointData><CellData><DataArray type="Float64" Name="pressure_Q0P0" format="ascii">\n')
    out += [_g(x) + "\n" for x in p[:nh + nt]]
    out.append('</DataArray><DataArray type="Int32" Name="region" format="ascii">\n')
    out += ["1\n"] * nh + ["2\n"] * nt
    out.append("</DataArray></CellData></Piece></UnstructuredGrid></VTKFile>\n")
    return "".join(out)


def parse_vtu(text: str) -> dict:
    """DataArray blocks by name (points under "points"), as float arrays."""
    import re
    blocks = {}
    for m in re.finditer(r'<DataArray type="(\w+)"(?: Name="(\w+)")?[^>]*>\n(.*?)</DataArray>', text, re.S):
        blocks[m.group(2) or "points"] = np.array(m.group(3).split(), dtype=np.float64)
    return blocks
