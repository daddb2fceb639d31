"""Mesh input for the device path: BABELSIM_MESH 3 files and seeded generators.

* read_mesh / write_mesh: the reference's text format (src/io/mesh_reader.cpp:44-111).
* hex_box: structured hexahedra on a box, optionally with warped vertices
  (the shape of the reference's test builders, tests/test_util.h:104-190).
* voronoi_cube: 3D Voronoi tessellation of jittered lattice sites clipped to
  the unit cube by mirror sites, built from the Delaunay tetrahedralisation.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class PolyMesh:
    vertices: np.ndarray        # (V,3)
    faces: list                 # vertex rings (or None when offsets/ids are given)
    owner: np.ndarray           # (F,)
    neighbour: np.ndarray       # (F,), -1 on boundary
    patch: np.ndarray           # (F,), -1 on interior
    patch_names: list = field(default_factory=list)
    patch_kinds: list = field(default_factory=list)
    offsets: np.ndarray = None  # (F+1,) flat ring storage, alternative to `faces`
    ids: np.ndarray = None

    @property
    def n_cells(self):
        return int(max(self.owner.max(), self.neighbour.max()) + 1)

    def flat(self):
        """(offsets, ids) of the face rings."""
        if self.offsets is not None:
            return self.offsets, self.ids
        off = np.concatenate([[0], np.cumsum([len(f) for f in self.faces])]).astype(np.int32)
        return off, np.concatenate(self.faces).astype(np.int32)

    def rings(self):
        if self.faces is not None:
            return self.faces
        return [self.ids[self.offsets[i]:self.offsets[i + 1]] for i in range(len(self.owner))]


def read_mesh(path) -> PolyMesh:
    """BABELSIM_MESH 3 reader."""
    tok = open(path).read().split()
    if tok[0] != "BABELSIM_MESH" or tok[1] != "3" or tok[2] != "vertices":
        raise ValueError(f"{path}: only BABELSIM_MESH version 3 is supported")
    nv = int(tok[3])
    pos = 4
    verts = np.array(tok[pos:pos + 3 * nv], dtype=np.float64).reshape(nv, 3)
    pos += 3 * nv
    if tok[pos] != "faces":
        raise ValueError(f"{path}: expected faces")
    nf = int(tok[pos + 1])
    pos += 2
    faces, owner, nbr, patch = [], np.empty(nf, np.int32), np.empty(nf, np.int32), np.empty(nf, np.int32)
    for f in range(nf):
        k = int(tok[pos + 1])
        owner[f], nbr[f], patch[f] = int(tok[pos + 2]), int(tok[pos + 3]), int(tok[pos + 4])
        faces.append(np.array(tok[pos + 5:pos + 5 + k], dtype=np.int64))
        pos += 5 + k
    if tok[pos] != "patches":
        raise ValueError(f"{path}: expected patches")
    npatch = int(tok[pos + 1])
    pos += 2
    names, kinds = [], []
    for _ in range(npatch):
        names.append(tok[pos + 1])
        kinds.append(tok[pos + 2])
        pos += 3
    return PolyMesh(verts, faces, owner, nbr, patch, names, kinds)


def write_mesh(path, mesh: PolyMesh):
    lines = ["BABELSIM_MESH 3", "vertices", str(len(mesh.vertices))]
    lines += [f"{x!r} {y!r} {z!r}" for x, y, z in mesh.vertices.tolist()]
    rings = mesh.rings()
    lines += ["faces", str(len(rings))]
    for f, ring in enumerate(rings):
        lines.append(f"face {len(ring)} {mesh.owner[f]} {mesh.neighbour[f]} {mesh.patch[f]} " +
                     " ".join(str(int(v)) for v in ring))
    lines += ["patches", str(len(mesh.patch_names))]
    for name, kind in zip(mesh.patch_names, mesh.patch_kinds):
        lines += ["patch", name, kind]
    lines.append("end")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def hex_box(nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), names=None, kinds=None, warp=None,
            flat=False) -> PolyMesh:
    """Structured hexahedra; cell (a,b,c) has index a + nx*(b + ny*c).

    Patches, in order: minus_x, plus_x, minus_y, plus_y, minus_z, plus_z (or
    ``names``).  ``warp(points)`` may move the vertices.  ``flat`` stores the face
    rings as offsets/ids arrays (large meshes) instead of a list.
    """
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    a, b, c = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    pts = np.stack([a.ravel(order="F"), b.ravel(order="F"), c.ravel(order="F")], axis=1).astype(float)
    verts = lo + (hi - lo) * pts / np.array([nx, ny, nz], float)
    if warp is not None:
        verts = warp(verts)

    def vid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    def cid(i, j, k):
        return i + nx * (j + ny * k)
    faces, own, nbr, pat = [], [], [], []

    def add(rings, o, n, p):
        faces.extend(list(rings))
        own.append(o)
        nbr.append(n)
        pat.append(p)
    # interior x faces between (i-1,j,k) and (i,j,k), i=1..nx-1
    I, J, K = np.meshgrid(np.arange(1, nx), np.arange(ny), np.arange(nz), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    rings_x = np.stack([vid(I, J, K), vid(I, J + 1, K), vid(I, J + 1, K + 1), vid(I, J, K + 1)], axis=1)
    I2, J2, K2 = np.meshgrid(np.arange(nx), np.arange(1, ny), np.arange(nz), indexing="ij")
    I2, J2, K2 = I2.ravel(), J2.ravel(), K2.ravel()
    rings_y = np.stack([vid(I2, J2, K2), vid(I2, J2, K2 + 1), vid(I2 + 1, J2, K2 + 1), vid(I2 + 1, J2, K2)], axis=1)
    I3, J3, K3 = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(1, nz), indexing="ij")
    I3, J3, K3 = I3.ravel(), J3.ravel(), K3.ravel()
    rings_z = np.stack([vid(I3, J3, K3), vid(I3 + 1, J3, K3), vid(I3 + 1, J3 + 1, K3), vid(I3, J3 + 1, K3)], axis=1)
    own_i = np.concatenate([cid(I - 1, J, K), cid(I2, J2 - 1, K2), cid(I3, J3, K3 - 1)])
    nbr_i = np.concatenate([cid(I, J, K), cid(I2, J2, K2), cid(I3, J3, K3)])
    ring_i = np.concatenate([rings_x, rings_y, rings_z]) if len(own_i) else np.zeros((0, 4), int)
    # boundary faces
    bo, br, bp = [], [], []
    jj, kk = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    jj, kk = jj.ravel(), kk.ravel()
    for side, i in ((0, 0), (1, nx)):
        br.append(np.stack([vid(i, jj, kk), vid(i, jj + 1, kk), vid(i, jj + 1, kk + 1), vid(i, jj, kk + 1)], axis=1))
        bo.append(cid(min(i, nx - 1), jj, kk))
        bp.append(np.full(len(jj), side))
    ii, kk = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    ii, kk = ii.ravel(), kk.ravel()
    for side, j in ((2, 0), (3, ny)):
        br.append(np.stack([vid(ii, j, kk), vid(ii, j, kk + 1), vid(ii + 1, j, kk + 1), vid(ii + 1, j, kk)], axis=1))
        bo.append(cid(ii, min(j, ny - 1), kk))
        bp.append(np.full(len(ii), side))
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    ii, jj = ii.ravel(), jj.ravel()
    for side, k in ((4, 0), (5, nz)):
        br.append(np.stack([vid(ii, jj, k), vid(ii + 1, jj, k), vid(ii + 1, jj + 1, k), vid(ii, jj + 1, k)], axis=1))
        bo.append(cid(ii, jj, min(k, nz - 1)))
        bp.append(np.full(len(ii), side))
    ring_b = np.concatenate(br)
    own_b = np.concatenate(bo)
    pat_b = np.concatenate(bp)
    rings = np.concatenate([ring_i, ring_b]).astype(np.int64)
    owner = np.concatenate([own_i, own_b]).astype(np.int32)
    neighbour = np.concatenate([nbr_i, np.full(len(own_b), -1)]).astype(np.int32)
    patch = np.concatenate([np.full(len(own_i), -1), pat_b]).astype(np.int32)
    names = names or ["minus_x", "plus_x", "minus_y", "plus_y", "minus_z", "plus_z"]
    kinds = kinds or ["generic"] * 6
    if flat:
        offsets = (4 * np.arange(len(rings) + 1)).astype(np.int32)
        return PolyMesh(verts, None, owner, neighbour, patch, list(names), list(kinds), offsets=offsets,
                        ids=rings.astype(np.int32).ravel())
    return PolyMesh(verts, list(rings), owner, neighbour, patch, list(names), list(kinds))


def channel(nx: int, ny: int, nz: int, length=2 * np.pi, height=2.0, width=np.pi, stretch=2.0, flat=True) -> PolyMesh:
    """Plane channel of hexahedra, wall-normal (y) spacing clustered at both walls by
    tanh stretching.  Patches: inlet, outlet, lower, upper (walls), front, back."""
    def warp(p):
        q = p.copy()
        eta = p[:, 1] / height * 2.0 - 1.0                    # [-1, 1]
        q[:, 1] = 0.5 * height * (1.0 + np.tanh(stretch * eta) / np.tanh(stretch))
        return q
    return hex_box(nx, ny, nz, (0.0, 0.0, 0.0), (length, height, width), warp=warp, flat=flat,
                   names=["inlet", "outlet", "lower", "upper", "front", "back"],
                   kinds=["inlet", "outlet", "wall", "wall", "symmetry", "symmetry"])


def cavity_2d(n: int) -> PolyMesh:
    """Unit-square lid-driven cavity, one cell thick (front/back symmetry planes)."""
    return hex_box(n, n, 1, (0, 0, 0), (1, 1, 1.0 / n),
                   names=["cavity_left", "cavity_right", "cavity_bottom", "lid", "front", "back"],
                   kinds=["wall", "wall", "wall", "wall", "symmetry", "symmetry"])


def warped_box(n: int, amplitude=0.08, seed=7) -> PolyMesh:
    """Unit cube of n^3 hexahedra with smoothly warped interior vertices (non-orthogonal, skewed)."""
    def warp(p):
        q = p.copy()
        inner = np.all((p > 1e-12) & (p < 1 - 1e-12), axis=1)
        x, y, z = p[:, 0], p[:, 1], p[:, 2]
        dx = amplitude * np.sin(np.pi * y) * np.sin(2 * np.pi * z) / n * 3
        dy = amplitude * np.sin(np.pi * z) * np.sin(2 * np.pi * x) / n * 3
        dz = amplitude * np.sin(np.pi * x) * np.sin(2 * np.pi * y) / n * 3
        q[inner, 0] += dx[inner]
        q[inner, 1] += dy[inner]
        q[inner, 2] += dz[inner]
        return q
    return hex_box(n, n, n, warp=warp,
                   names=["cavity_left", "cavity_right", "cavity_bottom", "lid", "front", "back"],
                   kinds=["wall"] * 6)




def cylinder_ogrid(n_theta: int, n_r: int, r0: float = 0.5, radius: float = 15.0, growth: float = 1.05,
                   dz: float = 0.1) -> PolyMesh:
    """O-grid of hexahedra around a circular cylinder (diameter 2 r0), one cell thick.

    Radial layers grow geometrically by `growth` from the cylinder to `radius`.
    Cell (a, b) has radial index a and angular index b (angles wrap around), index
    a + n_r b.  Patches: cylinder, inlet (outer faces with x < 0), outlet (outer
    faces with x >= 0), front, back.
    """
    a = np.arange(n_r + 1)
    h0 = (radius - r0) * (growth - 1.0) / (growth ** n_r - 1.0) if growth != 1.0 else (radius - r0) / n_r
    r = r0 + (h0 * (growth ** a - 1.0) / (growth - 1.0) if growth != 1.0 else h0 * a)
    th = 2.0 * np.pi * np.arange(n_theta) / n_theta
    A, B, Cz = np.meshgrid(np.arange(n_r + 1), np.arange(n_theta), np.arange(2), indexing="ij")
    A, B, Cz = A.ravel(order="F"), B.ravel(order="F"), Cz.ravel(order="F")
    verts = np.stack([r[A] * np.cos(th[B]), r[A] * np.sin(th[B]), dz * Cz], axis=1)

    def vid(i, j, k):
        return i + (n_r + 1) * ((j % n_theta) + n_theta * k)

    def cid(i, j):
        return i + n_r * (j % n_theta)
    # radial faces between (a-1, b) and (a, b)
    I, J = np.meshgrid(np.arange(1, n_r), np.arange(n_theta), indexing="ij")
    I, J = I.ravel(), J.ravel()
    rings_a = np.stack([vid(I, J, 0), vid(I, J + 1, 0), vid(I, J + 1, 1), vid(I, J, 1)], axis=1)
    own_a, nbr_a = cid(I - 1, J), cid(I, J)
    # angular faces between (a, b-1) and (a, b), wrapping at b = 0
    I2, J2 = np.meshgrid(np.arange(n_r), np.arange(n_theta), indexing="ij")
    I2, J2 = I2.ravel(), J2.ravel()
    rings_b = np.stack([vid(I2, J2, 0), vid(I2, J2, 1), vid(I2 + 1, J2, 1), vid(I2 + 1, J2, 0)], axis=1)
    own_b, nbr_b = cid(I2, J2 - 1), cid(I2, J2)
    # boundary faces
    jj = np.arange(n_theta)
    ring_cyl = np.stack([vid(0, jj, 0), vid(0, jj + 1, 0), vid(0, jj + 1, 1), vid(0, jj, 1)], axis=1)
    ring_out = np.stack([vid(n_r, jj, 0), vid(n_r, jj + 1, 0), vid(n_r, jj + 1, 1), vid(n_r, jj, 1)], axis=1)
    mid = 0.5 * (np.cos(th) + np.cos(th + 2 * np.pi / n_theta))
    out_patch = np.where(mid < 0.0, 1, 2)
    ii, jj2 = np.meshgrid(np.arange(n_r), np.arange(n_theta), indexing="ij")
    ii, jj2 = ii.ravel(), jj2.ravel()
    ring_front = np.stack([vid(ii, jj2, 0), vid(ii + 1, jj2, 0), vid(ii + 1, jj2 + 1, 0), vid(ii, jj2 + 1, 0)], axis=1)
    ring_back = np.stack([vid(ii, jj2, 1), vid(ii + 1, jj2, 1), vid(ii + 1, jj2 + 1, 1), vid(ii, jj2 + 1, 1)], axis=1)
    rings = np.concatenate([rings_a, rings_b, ring_cyl, ring_out, ring_front, ring_back]).astype(np.int64)
    owner = np.concatenate([own_a, own_b, cid(0, jj), cid(n_r - 1, jj), cid(ii, jj2), cid(ii, jj2)]).astype(np.int32)
    n_int = len(own_a) + len(own_b)
    neighbour = np.concatenate([nbr_a, nbr_b, np.full(len(owner) - n_int, -1)]).astype(np.int32)
    patch = np.concatenate([np.full(n_int, -1), np.zeros(n_theta), out_patch, np.full(len(ii), 3),
                            np.full(len(ii), 4)]).astype(np.int32)
    return PolyMesh(verts, list(rings), owner, neighbour, patch, ["cylinder", "inlet", "outlet", "front", "back"],
                    ["wall", "inlet", "outlet", "symmetry", "symmetry"])


def voronoi_cube(n: int, jitter: float = 0.3, seed: int = 20261007, names=None, kinds=None) -> PolyMesh:
    """Jittered-lattice Voronoi tessellation of the unit cube (see babelsim_b200.voronoi)."""
    from .voronoi import voronoi_cube as build
    return build(n, jitter, seed, names, kinds)


def concatenate(meshes) -> tuple:
    """Several independent meshes as one (the block-diagonal batch of bsg_simple_set_segments):
    vertices, cells, faces and patches of mesh k follow those of meshes 0..k-1, its patches
    named "<name>@k".  Returns (PolyMesh, cell_offsets, patch_offsets)."""
    verts, ids, own, nbr, pat, names, kinds = [], [], [], [], [], [], []
    v0 = c0 = p0 = 0
    cell_offsets, patch_offsets = [0], [0]
    for k, m in enumerate(meshes):
        o, i = m.flat()
        verts.append(np.asarray(m.vertices, np.float64))
        ids.append(np.asarray(i, np.int64) + v0)
        n = m.n_cells
        own.append(np.asarray(m.owner, np.int64) + c0)
        nb = np.asarray(m.neighbour, np.int64)
        nbr.append(np.where(nb >= 0, nb + c0, -1))
        pt = np.asarray(m.patch, np.int64)
        pat.append(np.where(pt >= 0, pt + p0, -1))
        names += [f"{nm}@{k}" for nm in m.patch_names]
        kinds += list(m.patch_kinds)
        v0 += len(m.vertices)
        c0 += n
        p0 += len(m.patch_names)
        cell_offsets.append(c0)
        patch_offsets.append(p0)
    # ring offsets: each mesh's offsets shifted by the rings before it
    flat_off = [np.zeros(1, np.int64)]
    base = 0
    for m in meshes:
        o, _ = m.flat()
        flat_off.append(np.asarray(o[1:], np.int64) + base)
        base += int(o[-1])
    pm = PolyMesh(np.concatenate(verts), None, np.concatenate(own).astype(np.int32),
                  np.concatenate(nbr).astype(np.int32), np.concatenate(pat).astype(np.int32), names, kinds,
                  offsets=np.concatenate(flat_off).astype(np.int32), ids=np.concatenate(ids).astype(np.int32))
    return pm, np.array(cell_offsets, np.int32), np.array(patch_offsets, np.int32)
