"""Seeded synthetic pipe meshes (tetrahedra) for the SIMPLE solver.

The reference solver reads ASCII OpenFOAM ``constant/polyMesh`` directories
(gpu/serial_cuda/foam_mesh_g2.hpp:55) whose patches follow the convention
wall ``patch_0_0``, inlet ``patch_2_0``, outlet ``patch_1_0``
(scripts/nodals_gpu_case.py:125-127).  Its pipe meshes are not shipped, so
this module generates stand-ins of the named shapes:

* cross-section: an O-grid made of a square core of ``k x k`` quads
  (``k = ntheta // 4``) surrounded by ``nr`` rings of ``ntheta`` quads that
  blend the core boundary onto the circle of radius ``R``;
* each quad is split into two triangles, the triangles are extruded through
  ``nz`` axial slabs into prisms, and every prism is split into 3 tetrahedra
  by the minimum-vertex-index rule, which splits each quadrilateral side
  face through its lowest-numbered vertex and therefore gives a conforming
  mesh (6 tetrahedra per quad and slab);
* interior nodes are jittered by a uniform +-``jitter`` fraction of the local
  spacing with a splitmix64 stream seeded per configuration; nodes on the
  wall keep their radius, nodes on the inlet/outlet keep their z.

Writers: ASCII polyMesh (faces ordered canonically, see ``canonical_faces``),
Gmsh MSH 2.2 with physical tags inlet=1, outlet=2, wall=3, volume=4
(turbulence/sst_gpu_v2/tools/msh2_to_hxt1.py:9-42), and binary HXT1.  The C++ readers build
the same canonical face order from either file, so both formats number the
velocity and pressure unknowns identically.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

MASK64 = (1 << 64) - 1

# patch order in the boundary file, as in the reference 40k pipe
PATCHES = ("patch_0_0", "patch_2_0", "patch_1_0")  # wall, inlet, outlet
MSH_TAG = {"patch_0_0": 3, "patch_2_0": 1, "patch_1_0": 2}
MSH_VOLUME_TAG = 4


def splitmix64_stream(seed: int, n: int) -> np.ndarray:
    """n outputs of splitmix64 (Steele, Lea, Flood 2014) as uint64."""
    with np.errstate(over="ignore"):
        gamma = np.uint64(0x9E3779B97F4A7C15)
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed & MASK64) + k * gamma
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, n: int) -> np.ndarray:
    """Uniform doubles in [0,1) from the top 53 bits of splitmix64."""
    return (splitmix64_stream(seed, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


@dataclass
class TetMesh:
    points: np.ndarray                 # (np, 3) float64
    tets: np.ndarray                   # (nc, 4) int32, positively oriented
    bfaces: np.ndarray                 # (nb, 3) int32 boundary triangles
    btag: np.ndarray                   # (nb,) int32: index into PATCHES
    meta: dict = field(default_factory=dict)

    @property
    def n_cells(self) -> int:
        return int(self.tets.shape[0])


def _cross_section(nr: int, ntheta: int, radius: float):
    """2-D O-grid nodes, quads (counter-clockwise) and boundary-edge flags."""
    if ntheta % 8 != 0 or ntheta < 8:
        raise ValueError("ntheta must be a positive multiple of 8")
    if nr < 1:
        raise ValueError("nr must be >= 1")
    k = ntheta // 4
    h = radius / (k / 2 + nr)
    a = 0.5 * k * h
    # core grid nodes
    idx = -np.ones((k + 1, k + 1), dtype=np.int64)
    xy = []
    for j in range(k + 1):
        for i in range(k + 1):
            idx[j, i] = len(xy)
            xy.append((-a + i * h, -a + j * h))
    # perimeter of the core, counter-clockwise starting at (-a,-a)
    perim = []
    for i in range(k):
        perim.append((0, i))
    for j in range(k):
        perim.append((j, k))
    for i in range(k, 0, -1):
        perim.append((k, i))
    for j in range(k, 0, -1):
        perim.append((j, 0))
    assert len(perim) == ntheta
    ring = -np.ones((nr + 1, ntheta), dtype=np.int64)
    for t, (j, i) in enumerate(perim):
        ring[0, t] = idx[j, i]
    xy = [list(p) for p in xy]
    sq = np.array([xy[ring[0, t]] for t in range(ntheta)])
    ang = np.arctan2(sq[:, 1], sq[:, 0])
    circ = np.stack([radius * np.cos(ang), radius * np.sin(ang)], axis=1)
    for r in range(1, nr + 1):
        lam = r / nr
        for t in range(ntheta):
            p = (1.0 - lam) * sq[t] + lam * circ[t]
            if r == nr:
                p = circ[t]
            ring[r, t] = len(xy)
            xy.append([p[0], p[1]])
    xy = np.asarray(xy, dtype=np.float64)
    quads = []
    for j in range(k):
        for i in range(k):
            quads.append((idx[j, i], idx[j, i + 1], idx[j + 1, i + 1], idx[j + 1, i]))
    for r in range(nr):
        for t in range(ntheta):
            t1 = (t + 1) % ntheta
            quads.append((ring[r, t], ring[r, t1], ring[r + 1, t1], ring[r + 1, t]))
    quads = np.asarray(quads, dtype=np.int64)
    on_wall = np.zeros(len(xy), dtype=bool)
    on_wall[ring[nr, :]] = True
    wall_edges = np.stack([ring[nr, :], ring[nr, (np.arange(ntheta) + 1) % ntheta]], axis=1)
    return xy, quads, on_wall, wall_edges


def _local_spacing_2d(xy, quads):
    h = np.full(len(xy), np.inf)
    for e in range(4):
        a = quads[:, e]
        b = quads[:, (e + 1) % 4]
        d = np.linalg.norm(xy[a] - xy[b], axis=1)
        np.minimum.at(h, a, d)
        np.minimum.at(h, b, d)
    return h


def _split_quads(xy, quads):
    """Two counter-clockwise triangles per quad through the shorter diagonal."""
    d02 = np.linalg.norm(xy[quads[:, 0]] - xy[quads[:, 2]], axis=1)
    d13 = np.linalg.norm(xy[quads[:, 1]] - xy[quads[:, 3]], axis=1)
    use02 = d02 <= d13
    t1 = np.where(use02[:, None], quads[:, [0, 1, 2]], quads[:, [0, 1, 3]])
    t2 = np.where(use02[:, None], quads[:, [0, 2, 3]], quads[:, [1, 2, 3]])
    return np.concatenate([t1, t2], axis=0)


def _prism_tets(bot: np.ndarray, top: np.ndarray) -> np.ndarray:
    """Split prisms (bot[i], top[i]) into 3 tets each by the min-index rule."""
    n = bot.shape[0]
    v = np.concatenate([bot, top], axis=1)  # v0 v1 v2 | v3 v4 v5 with v(i+3) above v(i)
    # the 6 prism symmetries that keep the structure: rotate the triangle, swap top/bottom
    perms = np.array([
        [0, 1, 2, 3, 4, 5], [1, 2, 0, 4, 5, 3], [2, 0, 1, 5, 3, 4],
        [3, 5, 4, 0, 2, 1], [4, 3, 5, 1, 0, 2], [5, 4, 3, 2, 1, 0],
    ])
    which = np.argmin(v, axis=1)  # vertex holding the global minimum
    p = perms[which]
    w = np.take_along_axis(v, p, axis=1)
    v0, v1, v2, v3, v4, v5 = (w[:, i] for i in range(6))
    diag15 = np.minimum(v1, v5) < np.minimum(v2, v4)
    t = np.empty((n, 3, 4), dtype=np.int64)
    t[:, 0] = np.where(diag15[:, None], np.stack([v0, v1, v2, v5], 1), np.stack([v0, v1, v2, v4], 1))
    t[:, 1] = np.where(diag15[:, None], np.stack([v0, v1, v5, v4], 1), np.stack([v0, v4, v2, v5], 1))
    t[:, 2] = np.stack([v0, v4, v5, v3], 1)
    return t.reshape(-1, 4)


def _orient(points: np.ndarray, tets: np.ndarray) -> np.ndarray:
    x = points[tets]
    det = np.einsum("ij,ij->i", np.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]), x[:, 3] - x[:, 0])
    out = tets.copy()
    neg = det < 0
    out[neg, 1], out[neg, 2] = tets[neg, 2], tets[neg, 1]
    if np.any(det == 0):
        raise RuntimeError("degenerate tetrahedron generated")
    return out


def pipe_mesh(nr: int = 8, ntheta: int = 24, nz: int = 35, radius: float = 0.5,
              length: float = 10.0, jitter: float = 0.05, seed: int = 0, bend_deg: float = 0.0) -> TetMesh:
    """Circular pipe from the inlet disk at z=0 to the outlet at axial length
    `length`: straight along +z, or (bend_deg > 0) with its axis bent in the
    x-z plane along a circular arc that turns by bend_deg over the length (the
    cross-sections stay normal to the axis; the inlet disk is unchanged)."""
    xy, quads, on_wall, wall_edges = _cross_section(nr, ntheta, radius)
    h2 = _local_spacing_2d(xy, quads)
    tri = _split_quads(xy, quads)
    n2 = len(xy)
    nl = nz + 1
    z = np.linspace(0.0, length, nl)
    pts = np.zeros((n2 * nl, 3))
    pts[:, 0] = np.tile(xy[:, 0], nl)
    pts[:, 1] = np.tile(xy[:, 1], nl)
    pts[:, 2] = np.repeat(z, n2)
    if jitter > 0.0:
        u = uniform01(seed, 3 * len(pts)).reshape(-1, 3) * 2.0 - 1.0
        hxy = np.tile(h2, nl)
        hz = length / nz
        free_xy = ~np.tile(on_wall, nl)
        layer = np.repeat(np.arange(nl), n2)
        free_z = (layer > 0) & (layer < nz)
        pts[:, 0] += np.where(free_xy, jitter * hxy * u[:, 0], 0.0)
        pts[:, 1] += np.where(free_xy, jitter * hxy * u[:, 1], 0.0)
        pts[:, 2] += np.where(free_z, jitter * hz * u[:, 2], 0.0)
    if bend_deg > 0.0:
        # axis point at arc length z: (Rc (1 - cos phi), 0, Rc sin phi), phi = z / Rc;
        # the section's x direction turns with the axis: (cos phi, 0, -sin phi)
        rc = length / np.deg2rad(bend_deg)
        if rc <= radius:
            raise ValueError("bend radius must exceed the pipe radius")
        phi = pts[:, 2] / rc
        x = pts[:, 0].copy()
        pts[:, 0] = rc * (1.0 - np.cos(phi)) + x * np.cos(phi)
        pts[:, 2] = rc * np.sin(phi) - x * np.sin(phi)
    tets = []
    for s in range(nz):
        tets.append(_prism_tets(tri + s * n2, tri + (s + 1) * n2))
    tets = _orient(pts, np.concatenate(tets, axis=0)).astype(np.int32)
    # boundary triangles
    inlet = tri.copy()
    outlet = tri + nz * n2
    wall = []
    for s in range(nz):
        a = wall_edges[:, 0] + s * n2
        b = wall_edges[:, 1] + s * n2
        c = wall_edges[:, 1] + (s + 1) * n2
        d = wall_edges[:, 0] + (s + 1) * n2
        quad = np.stack([a, b, c, d], axis=1)
        # split through the quad's minimum vertex (matches the prism rule)
        m = np.argmin(quad, axis=1)
        q = np.take_along_axis(quad, (m[:, None] + np.arange(4)[None, :]) % 4, axis=1)
        wall.append(np.stack([q[:, 0], q[:, 1], q[:, 2]], 1))
        wall.append(np.stack([q[:, 0], q[:, 2], q[:, 3]], 1))
    wall = np.concatenate(wall, axis=0)
    bfaces = np.concatenate([wall, inlet, outlet], axis=0).astype(np.int32)
    btag = np.concatenate([np.zeros(len(wall)), np.ones(len(inlet)), 2 * np.ones(len(outlet))]).astype(np.int32)
    meta = dict(nr=nr, ntheta=ntheta, nz=nz, radius=radius, length=length, jitter=jitter, seed=seed, bend_deg=bend_deg)
    return TetMesh(points=pts, tets=tets, bfaces=bfaces, btag=btag, meta=meta)


# ---------------------------------------------------------------------------
# canonical face order (shared with the C++ readers)
# ---------------------------------------------------------------------------

def canonical_faces(m: TetMesh):
    """Faces in the canonical order used by every reader of this package.

    Internal faces sorted by (owner, neighbour) with owner < neighbour, then
    boundary faces grouped by patch in ``PATCHES`` order and sorted by
    (owner, sorted vertex triple).  Each face is oriented with its normal
    pointing out of the owner cell.  Returns (faces[nf,3], owner[nf],
    neighbour[ni], patch_start[3], patch_size[3]).
    """
    nc = m.n_cells
    local = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])
    f = m.tets[:, local].reshape(-1, 3).astype(np.int64)
    cell = np.repeat(np.arange(nc, dtype=np.int64), 4)
    fs = np.sort(f, axis=1)
    key = (fs[:, 0] * (1 << 21) + fs[:, 1]) * (1 << 21) + fs[:, 2]
    if m.points.shape[0] >= (1 << 21):
        raise ValueError("canonical face keys support < 2^21 points")
    order = np.lexsort((cell, key))
    ks = key[order]
    same_next = np.concatenate([ks[1:] == ks[:-1], [False]])
    same_prev = np.concatenate([[False], ks[1:] == ks[:-1]])
    first = order[same_next]
    second = order[np.where(same_next)[0] + 1]
    own_i = cell[first]
    nei_i = cell[second]
    swap = own_i > nei_i
    own_i, nei_i = np.where(swap, nei_i, own_i), np.where(swap, own_i, nei_i)
    tri_i = fs[first]
    io = np.lexsort((nei_i, own_i))
    own_i, nei_i, tri_i = own_i[io], nei_i[io], tri_i[io]
    single = order[~same_next & ~same_prev]
    bkey = key[single]
    bcell = cell[single]
    btri = fs[single]
    # tag lookup
    bs = np.sort(m.bfaces.astype(np.int64), axis=1)
    tkey = (bs[:, 0] * (1 << 21) + bs[:, 1]) * (1 << 21) + bs[:, 2]
    tord = np.argsort(tkey)
    pos = np.searchsorted(tkey[tord], bkey)
    if np.any(pos >= len(tkey)) or np.any(tkey[tord][np.minimum(pos, len(tkey) - 1)] != bkey):
        raise ValueError("boundary face without a tag")
    btag = m.btag[tord][pos]
    if len(single) != len(m.bfaces):
        raise ValueError("tagged boundary triangles do not match the mesh boundary")
    bo = np.lexsort((btri[:, 2], btri[:, 1], btri[:, 0], bcell, btag))
    bcell, btri, btag = bcell[bo], btri[bo], btag[bo]
    faces = np.concatenate([tri_i, btri], axis=0)
    owner = np.concatenate([own_i, bcell])
    # orient each face out of its owner: normal . (face centroid - cell centroid) > 0
    P = m.points
    a, b, c = P[faces[:, 0]], P[faces[:, 1]], P[faces[:, 2]]
    n = np.cross(b - a, c - a)
    cc = P[m.tets[owner]].mean(axis=1)
    fc = (a + b + c) / 3.0
    flip = np.einsum("ij,ij->i", n, fc - cc) < 0
    faces[flip, 1], faces[flip, 2] = faces[flip, 2].copy(), faces[flip, 1].copy()
    counts = np.bincount(btag, minlength=len(PATCHES))
    start = len(tri_i) + np.concatenate([[0], np.cumsum(counts)[:-1]])
    return faces.astype(np.int32), owner.astype(np.int32), nei_i.astype(np.int32), start, counts


_FOAM_HEADER = """/*--------------------------------*- C++ -*----------------------------------*\\
  nodals_b200 synthetic pipe mesh
\\*---------------------------------------------------------------------------*/
FoamFile
{{
    format      ascii;
    class       {cls};
    location    "constant/polyMesh";
    object      {obj};
}}
// * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * //

"""


def _write_list(path: Path, cls: str, obj: str, body_lines, n: int):
    with open(path, "w") as f:
        f.write(_FOAM_HEADER.format(cls=cls, obj=obj))
        f.write(f"{n}\n(\n")
        f.write(body_lines)
        f.write(")\n")


def write_polymesh(m: TetMesh, directory: str | os.PathLike) -> Path:
    """Write ``directory/constant/polyMesh`` (or ``directory`` if it already ends in polyMesh)."""
    d = Path(directory)
    if d.name != "polyMesh":
        d = d / "constant" / "polyMesh"
    d.mkdir(parents=True, exist_ok=True)
    faces, owner, neighbour, start, counts = canonical_faces(m)
    pts = "\n".join(f"({x:.17g} {y:.17g} {z:.17g})" for x, y, z in m.points) + "\n"
    _write_list(d / "points", "vectorField", "points", pts, len(m.points))
    fl = "\n".join(f"3({a} {b} {c})" for a, b, c in faces) + "\n"
    _write_list(d / "faces", "faceList", "faces", fl, len(faces))
    _write_list(d / "owner", "labelList", "owner", "\n".join(map(str, owner)) + "\n", len(owner))
    _write_list(d / "neighbour", "labelList", "neighbour", "\n".join(map(str, neighbour)) + "\n", len(neighbour))
    with open(d / "boundary", "w") as f:
        f.write(_FOAM_HEADER.format(cls="polyBoundaryMesh", obj="boundary"))
        f.write(f"{len(PATCHES)}\n(\n")
        for name, s, n in zip(PATCHES, start, counts):
            f.write(f"    {name}\n    {{\n        type            patch;\n        physicalType    patch;\n")
            f.write(f"        nFaces          {int(n)};\n        startFace       {int(s)};\n    }}\n")
        f.write(")\n")
    return d


def write_msh2(m: TetMesh, path: str | os.PathLike) -> Path:
    """Gmsh MSH 2.2 ASCII: tagged boundary triangles then tetrahedra (1-based ids)."""
    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    with open(p, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n")
        f.write("$PhysicalNames\n4\n2 1 \"inlet\"\n2 2 \"outlet\"\n2 3 \"wall\"\n3 4 \"fluid\"\n$EndPhysicalNames\n")
        f.write(f"$Nodes\n{len(m.points)}\n")
        f.write("\n".join(f"{i + 1} {x:.17g} {y:.17g} {z:.17g}" for i, (x, y, z) in enumerate(m.points)))
        f.write("\n$EndNodes\n")
        ne = len(m.bfaces) + len(m.tets)
        f.write(f"$Elements\n{ne}\n")
        lines = []
        e = 1
        for tri, t in zip(m.bfaces, m.btag):
            tag = MSH_TAG[PATCHES[t]]
            lines.append(f"{e} 2 2 {tag} {tag} {tri[0] + 1} {tri[1] + 1} {tri[2] + 1}")
            e += 1
        for tet in m.tets:
            lines.append(f"{e} 4 2 {MSH_VOLUME_TAG} {MSH_VOLUME_TAG} {tet[0] + 1} {tet[1] + 1} {tet[2] + 1} {tet[3] + 1}")
            e += 1
        f.write("\n".join(lines))
        f.write("\n$EndElements\n")
    return p


# Binary HXT1, the mixed hex/tet mesh format of the reference's hybrid and
# SST solvers (gpu/serial_cuda/hybrid_hxt1/hxt1_mesh.hpp:19-103), written
# here for pure-tet meshes as the reference's converter does
# (turbulence/sst_gpu_v2/tools/msh2_to_hxt1.py: positively oriented tets,
# inlet and outlet tet records, no wall records).
HXT1_MAGIC = b"HXT1BIN1"
HXT1_TET_FACE = ((1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1))  # face opposite local vertex lf


def _det3_cols(a, b, c):
    """Determinant of the 3x3 matrices with columns a, b, c (rows of (n, 3) arrays)."""
    return (a[:, 0] * (b[:, 1] * c[:, 2] - b[:, 2] * c[:, 1])
            - b[:, 0] * (a[:, 1] * c[:, 2] - a[:, 2] * c[:, 1])
            + c[:, 0] * (a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1]))


def write_hxt1(m: TetMesh, path: str | os.PathLike) -> Path:
    """HXT1 version 1 for a tetrahedral mesh: points; tets with a positive
    Jacobian (vertices 2 and 3 swapped otherwise); per tet the 8 velocity
    unknowns (4 vertices, then the bubbles of the faces opposite vertices
    0..3, a face's bubble numbered n_points + the rank of its sorted vertex
    triple); pressure ids 0..nt-1; geometry (volume, squared longest edge,
    det J, J^-1 row-major, J = [X1-X0 | X2-X0 | X3-X0]); the inlet and
    outlet faces as (tet, local face, bubble) records in boundary-list
    order.  All other counts are zero."""
    pts = np.ascontiguousarray(m.points, dtype=np.float64)
    tets = np.array(m.tets, dtype=np.int32)
    nv, nt = len(pts), len(tets)
    x = pts[tets]
    det = _det3_cols(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], x[:, 3] - x[:, 0])
    flip = det < 0
    tets[flip, 2], tets[flip, 3] = tets[flip, 3].copy(), tets[flip, 2].copy()
    x = pts[tets]
    e1, e2, e3 = x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]
    det = _det3_cols(e1, e2, e3)
    # J^-1 = adj(J) / det; with J's columns e1, e2, e3 the rows of J^-1 are
    # e2 x e3, e3 x e1, e1 x e2 divided by det
    inv = np.stack((np.cross(e2, e3), np.cross(e3, e1), np.cross(e1, e2)), axis=1) / det[:, None, None]
    h2 = np.zeros(nt)
    for a in range(4):
        for b in range(a + 1, 4):
            d = x[:, a] - x[:, b]
            h2 = np.maximum(h2, np.einsum("ij,ij->i", d, d))
    geom = np.column_stack((det / 6.0, h2, det, inv.reshape(nt, 9)))
    keys = np.sort(tets[:, np.asarray(HXT1_TET_FACE)], axis=2).reshape(-1, 3)
    uniq, rank = np.unique(keys, axis=0, return_inverse=True)
    bubble = (nv + rank.reshape(nt, 4)).astype(np.int32)
    tvel = np.concatenate((tets, bubble), axis=1)
    lookup = {tuple(k): (i // 4, i % 4) for i, k in enumerate(map(tuple, keys))}

    def records(tag):
        out = []
        for tri in m.bfaces[m.btag == tag]:
            c, lf = lookup[tuple(sorted(int(v) for v in tri))]
            out.append((c, lf, int(bubble[c, lf])))
        return np.asarray(out, dtype=np.int32).reshape(-1, 3)
    rin, rout = records(PATCHES.index("patch_2_0")), records(PATCHES.index("patch_1_0"))
    header = (nv, 0, nt, 0, len(uniq), nv + len(uniq), nt, 0, 0, 0, len(rin), 0, len(rout))
    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    with open(p, "wb") as f:
        f.write(HXT1_MAGIC + np.asarray([1, 0], dtype="<u4").tobytes() + np.asarray(header, dtype="<u8").tobytes())
        for a in (pts, tets, tvel, np.arange(nt, dtype=np.int32), geom, rin, rout):
            f.write(np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes())
    return p


# ---------------------------------------------------------------------------
# hybrid hex/tet pipes (the mixed meshes of the reference's HXT solvers)
# ---------------------------------------------------------------------------
HXT1_HEX_FACE = ((0, 1, 2, 3), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7))


@dataclass
class HybridMesh:
    """Mixed mesh in the array form the reference's HXT1 preparer reads
    (gpu/serial_cuda/hybrid_hxt1/prepare_hxt1.py: HXT0 arrays)."""
    points: np.ndarray                # (np, 3)
    hexes: np.ndarray                 # (nh, 8): bottom quad counter-clockwise, then the top quad
    tets: np.ndarray                  # (nt, 4) positively oriented
    interface_quads: np.ndarray       # (ni, 4) hex faces shared with the tet region
    interface_triangles: np.ndarray   # (ni, 2, 3) the two tet faces covering each
    wall_quads: np.ndarray
    inlet_hex_quads: np.ndarray
    inlet_tet_triangles: np.ndarray
    outlet_hex_quads: np.ndarray
    outlet_tet_triangles: np.ndarray
    meta: dict = field(default_factory=dict)

    def arrays(self) -> dict:
        return {k: getattr(self, k) for k in ("points", "hexes", "tets", "interface_quads", "interface_triangles",
                                              "wall_quads", "inlet_hex_quads", "inlet_tet_triangles",
                                              "outlet_hex_quads", "outlet_tet_triangles")}


def hybrid_pipe(nr: int = 4, ntheta: int = 16, nz: int = 40, radius: float = 0.5, length: float = 10.0) -> HybridMesh:
    """Straight pipe with the cross-section of ``pipe_mesh``: its ``nr`` rings
    of quads are extruded into hexahedra (they carry the wall), its square
    core into prisms split into tetrahedra by the minimum-vertex rule.  The
    hex/tet interface is the core boundary: each of its quads is a hex face
    covered by two tet faces.  No jitter, so every face is planar."""
    xy, quads, _on_wall, _ = _cross_section(nr, ntheta, radius)
    k = ntheta // 4
    core, ring = quads[: k * k], quads[k * k:]
    # hex bottoms counter-clockwise seen from +z (positive Jacobian)
    e1, e2 = xy[ring[:, 1]] - xy[ring[:, 0]], xy[ring[:, 3]] - xy[ring[:, 0]]
    cw = e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0] < 0
    ring = np.where(cw[:, None], ring[:, [0, 3, 2, 1]], ring)
    n2, nl = len(xy), nz + 1
    z = np.linspace(0.0, length, nl)
    pts = np.zeros((n2 * nl, 3))
    pts[:, 0] = np.tile(xy[:, 0], nl)
    pts[:, 1] = np.tile(xy[:, 1], nl)
    pts[:, 2] = np.repeat(z, n2)
    hexes = np.concatenate([np.concatenate([ring + s * n2, ring + (s + 1) * n2], axis=1) for s in range(nz)])
    tri = _split_quads(xy, core)
    tets = _orient(pts, np.concatenate([_prism_tets(tri + s * n2, tri + (s + 1) * n2) for s in range(nz)]))
    faces = {}
    for c, t in enumerate(tets):
        for f in HXT1_TET_FACE:
            tri3 = tuple(int(t[i]) for i in f)
            faces[tuple(sorted(tri3))] = tri3
    # interface: the inner side faces of the first ring's hexes
    # inner edge of a first-ring quad: its two vertices on the core boundary
    core_nodes = set(int(v) for v in core.reshape(-1))
    ring0 = ring[:ntheta]
    iq, it = [], []
    for s in range(nz):
        for q in ring0:
            a, b = [int(v) + s * n2 for v in q if int(v) in core_nodes]
            quad = (a, b, b + n2, a + n2)
            for t1, t2 in (((quad[0], quad[1], quad[2]), (quad[0], quad[2], quad[3])),
                           ((quad[0], quad[1], quad[3]), (quad[1], quad[2], quad[3]))):
                k1, k2 = tuple(sorted(t1)), tuple(sorted(t2))
                if k1 in faces and k2 in faces:
                    iq.append(quad)
                    it.append((faces[k1], faces[k2]))
                    break
            else:
                raise RuntimeError("interface quad not covered by two tet faces")
    wall_nodes = set(int(v) for v in ring[-ntheta:].reshape(-1)) - set(int(v) for v in ring[-2 * ntheta:-ntheta].reshape(-1)) \
        if nr > 1 else set(int(v) for v in ring.reshape(-1)) - core_nodes
    wall = []
    for s in range(nz):
        for q in ring[-ntheta:]:
            a, b = [int(v) + s * n2 for v in q if int(v) in wall_nodes]
            wall.append((a, b, b + n2, a + n2))
    as32 = lambda a, w: np.asarray(a, dtype=np.int32).reshape(-1, *w)
    return HybridMesh(
        points=pts, hexes=as32(hexes, (8,)), tets=as32(tets, (4,)),
        interface_quads=as32(iq, (4,)), interface_triangles=as32(it, (2, 3)), wall_quads=as32(wall, (4,)),
        inlet_hex_quads=as32(ring, (4,)), inlet_tet_triangles=as32(tri, (3,)),
        outlet_hex_quads=as32(ring + nz * n2, (4,)), outlet_tet_triangles=as32(tri + nz * n2, (3,)),
        meta=dict(nr=nr, ntheta=ntheta, nz=nz, radius=radius, length=length))


_HEX_SIGN = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                      [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)


def _face_table(cells: np.ndarray, faces) -> tuple:
    """Sorted vertex keys of every local face (cell-major), the unique keys in
    lexicographic order and each local face's rank among them."""
    k = np.sort(cells[:, np.asarray(faces)], axis=2).reshape(-1, len(faces[0]))
    uniq, inv, cnt = np.unique(k, axis=0, return_inverse=True, return_counts=True)
    if np.any(cnt > 2):
        raise ValueError("non-manifold face")
    return k, uniq, inv.reshape(len(cells), len(faces)), cnt


def _locate(uniq: np.ndarray, rank: np.ndarray, cnt: np.ndarray, recs: np.ndarray, what: str) -> np.ndarray:
    """(cell, local face, rank) of the faces of recs (vertex lists), each of
    which must have exactly one owner."""
    recs = np.asarray(recs, dtype=np.int64).reshape(-1, uniq.shape[1])
    if len(recs) == 0:
        return np.zeros((0, 3), dtype=np.int64)
    keys = np.sort(recs, axis=1)
    # row of each key in uniq: as big-endian unsigned bytes, the byte order
    # of a key is its lexicographic order, so a void view searches sorted
    big = np.dtype(">u4")
    vu = np.ascontiguousarray(uniq.astype(big)).view(np.dtype((np.void, 4 * uniq.shape[1]))).ravel()
    vk = np.ascontiguousarray(keys.astype(big)).view(vu.dtype).ravel()
    pos = np.searchsorted(vu, vk)
    if np.any(pos >= len(vu)) or np.any(vu[np.minimum(pos, len(vu) - 1)] != vk):
        raise ValueError(f"{what} face not found in the mesh")
    if np.any(cnt[pos] != 1):
        raise ValueError(f"{what} face owner count != 1")
    flat = np.full(len(uniq), -1, dtype=np.int64)
    flat[rank.ravel()] = np.arange(rank.size)
    owner = flat[pos]  # the single owner's (cell * nfaces + local face)
    nf = rank.shape[1]
    return np.stack((owner // nf, owner % nf, pos), axis=1)


def write_hxt1_hybrid(m: HybridMesh, path: str | os.PathLike) -> Path:
    """HXT1 version 1 of a mixed mesh, laid out as the reference's preparer
    writes it (gpu/serial_cuda/hybrid_hxt1/prepare_hxt1.py:110-246): the face
    bubbles of hex faces numbered n_points + the rank of the sorted vertex
    quadruple, then those of tet faces after them; per hex the 8 vertices and
    6 face bubbles, per tet 4 vertices and 4; pressure ids hexes then tets;
    hex geometry (volume = sum of det J at the 2x2x2 Gauss points, squared
    longest vertex distance, the 8 det J, the 8 J^-1 row-major), tet geometry
    (volume, squared longest edge, det J, J^-1); interface records (hex cell,
    face, bubble, then the two tets'); wall, inlet and outlet records (cell,
    local face, bubble) in the order of the mesh's lists."""
    pts = np.ascontiguousarray(m.points, dtype=np.float64)
    hexes = np.ascontiguousarray(m.hexes, dtype=np.int32)
    tets = np.ascontiguousarray(m.tets, dtype=np.int32)
    nv, nh, nt = len(pts), len(hexes), len(tets)
    _, hu, hrank, hcnt = _face_table(hexes, HXT1_HEX_FACE)
    _, tu, trank, tcnt = _face_table(tets, HXT1_TET_FACE)
    nhf, ntf = len(hu), len(tu)
    hvel = np.concatenate((hexes, nv + hrank), axis=1).astype(np.int32)
    tvel = np.concatenate((tets, nv + nhf + trank), axis=1).astype(np.int32)
    iq = np.asarray(m.interface_quads).reshape(-1, 4)
    itr = np.asarray(m.interface_triangles).reshape(-1, 2, 3)
    if len(iq) != len(itr):
        raise ValueError("interface quad/triangle record mismatch")
    hrec = _locate(hu, hrank, hcnt, iq, "interface hex")
    t0 = _locate(tu, trank, tcnt, itr[:, 0], "interface tet")
    t1 = _locate(tu, trank, tcnt, itr[:, 1], "interface tet")
    off_h, off_t = np.array([0, 0, nv]), np.array([0, 0, nv + nhf])
    irec = np.concatenate((hrec + off_h, t0 + off_t, t1 + off_t), axis=1).astype(np.int32)
    recs = [_locate(hu, hrank, hcnt, m.wall_quads, "wall") + off_h,
            _locate(hu, hrank, hcnt, m.inlet_hex_quads, "inlet hex") + off_h,
            _locate(tu, trank, tcnt, m.inlet_tet_triangles, "inlet tet") + off_t,
            _locate(hu, hrank, hcnt, m.outlet_hex_quads, "outlet hex") + off_h,
            _locate(tu, trank, tcnt, m.outlet_tet_triangles, "outlet tet") + off_t]
    recs = [r.astype(np.int32) for r in recs]
    # hex geometry at the 2x2x2 Gauss points, xi slowest
    x = pts[hexes]  # (nh, 8, 3)
    g = 1.0 / np.sqrt(3.0)
    dets, invs = [], []
    for xi in (-g, g):
        for eta in (-g, g):
            for zeta in (-g, g):
                sx, sy, sz = _HEX_SIGN[:, 0], _HEX_SIGN[:, 1], _HEX_SIGN[:, 2]
                dxi = 0.125 * sx * (1.0 + sy * eta) * (1.0 + sz * zeta)
                deta = 0.125 * sy * (1.0 + sx * xi) * (1.0 + sz * zeta)
                dzeta = 0.125 * sz * (1.0 + sx * xi) * (1.0 + sy * eta)
                # J[:, i, j] = d x_i / d xi_j, each column one 8-term product
                J = np.stack((np.matmul(dxi, x), np.matmul(deta, x), np.matmul(dzeta, x)), axis=2)
                dets.append(np.linalg.det(J))
                invs.append(np.linalg.inv(J).reshape(nh, 9))
    dets = np.stack(dets, axis=1) if nh else np.zeros((0, 8))
    invs = np.concatenate(invs, axis=1) if nh else np.zeros((0, 72))
    h2h = np.zeros(nh)
    for a in range(8):
        for b in range(a + 1, 8):
            dd = x[:, a] - x[:, b]
            h2h = np.maximum(h2h, dd[:, 0] * dd[:, 0] + dd[:, 1] * dd[:, 1] + dd[:, 2] * dd[:, 2])
    vol = np.zeros(nh)
    for k in range(8):  # summed in Gauss-point order
        vol = vol + dets[:, k]
    hgeom = np.column_stack((vol, h2h, dets, invs)) if nh else np.zeros((0, 82))
    y = pts[tets]
    Jt = np.stack((y[:, 1] - y[:, 0], y[:, 2] - y[:, 0], y[:, 3] - y[:, 0]), axis=2)  # columns
    dt = np.linalg.det(Jt) if nt else np.zeros(0)
    it_ = np.linalg.inv(Jt).reshape(nt, 9) if nt else np.zeros((0, 9))
    h2t = np.zeros(nt)
    for a in range(4):
        for b in range(a + 1, 4):
            dd = y[:, a] - y[:, b]
            h2t = np.maximum(h2t, np.einsum("ij,ij->i", dd, dd))
    tgeom = np.column_stack((dt / 6.0, h2t, dt, it_)) if nt else np.zeros((0, 12))
    if nh and np.min(dets) <= 0 or nt and np.min(dt) <= 0:
        raise ValueError("non-positive Jacobian")
    header = (nv, nh, nt, nhf, ntf, nv + nhf + ntf, nh + nt, len(irec), *(len(r) for r in recs))
    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    with open(p, "wb") as f:
        f.write(HXT1_MAGIC + np.asarray([1, 0], dtype="<u4").tobytes() + np.asarray(header, dtype="<u8").tobytes())
        for a in (pts, hexes, tets, hvel, tvel, np.arange(nh, dtype=np.int32), np.arange(nh, nh + nt, dtype=np.int32),
                  hgeom, tgeom, irec, *recs):
            f.write(np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes())
    return p


def write_hxt0(m: HybridMesh, path: str | os.PathLike) -> Path:
    """The HXT0 ``.npz`` the reference's HXT1 preparer takes as input."""
    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    np.savez(p, **m.arrays())
    return p


# named workloads: (nr, ntheta, nz, radius, length, jitter, seed)
CONFIGS = {
    # ~40k-tet pipe, Re=20 (8 rings x 24 sectors x 35 slabs)
    "pipe40k": dict(nr=8, ntheta=24, nz=35, radius=0.5, length=10.0, jitter=0.05, seed=0),
    # ~1M-tet pipe, Re=100 (24 rings x 72 sectors x 100 slabs)
    "pipe1m": dict(nr=24, ntheta=72, nz=100, radius=0.5, length=10.0, jitter=0.05, seed=1),
    # ~380k-tet pipe for kernel profiling (fine CSR ~300 MB > L2)
    "pipe400k": dict(nr=16, ntheta=48, nz=70, radius=0.5, length=10.0, jitter=0.05, seed=2),
    # small parity meshes
    "pipe_tiny": dict(nr=2, ntheta=8, nz=6, radius=0.5, length=3.0, jitter=0.05, seed=7),
    "pipe_small": dict(nr=3, ntheta=16, nz=12, radius=0.5, length=5.0, jitter=0.05, seed=3),
}


def named(name: str) -> TetMesh:
    return pipe_mesh(**CONFIGS[name])


# The learned stage's pipe family: members 0..63 train, 64..79 are held out.
# Radius U[0.4, 0.6], length U[8, 12], axial bend U[0, 60] degrees, Re
# U[10, 200], ~200k tets (12 rings x 40 sectors + 10 x 10 core, 58 slabs),
# +-5 % jitter; every draw from the splitmix64 stream of the member.
FAMILY_TRAIN, FAMILY_HELD_OUT = 64, 16


def family_member(index: int):
    """(mesh, Re, parameters) of member `index` of the learned stage's family."""
    u = uniform01(0xC4F40000 + int(index), 4)
    prm = dict(radius=0.4 + 0.2 * float(u[0]), length=8.0 + 4.0 * float(u[1]), bend_deg=60.0 * float(u[2]))
    re = 10.0 + 190.0 * float(u[3])
    mesh = pipe_mesh(nr=12, ntheta=40, nz=58, jitter=0.05, seed=1000 + int(index), **prm)
    return mesh, re, dict(prm, re=re)


if __name__ == "__main__":  # pragma: no cover - convenience CLI
    import argparse

    ap = argparse.ArgumentParser(description="write a synthetic pipe mesh")
    ap.add_argument("config", choices=sorted(CONFIGS))
    ap.add_argument("--polymesh", help="case directory for constant/polyMesh")
    ap.add_argument("--msh", help="MSH 2.2 output path")
    ns = ap.parse_args()
    mesh = named(ns.config)
    print(f"cells={mesh.n_cells} points={len(mesh.points)} bfaces={len(mesh.bfaces)}")
    if ns.polymesh:
        print(write_polymesh(mesh, ns.polymesh))
    if ns.msh:
        print(write_msh2(mesh, ns.msh))
