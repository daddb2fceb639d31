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


def hex_box(nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), names=None, kinds=None, warp=None) -> PolyMesh:
    """Structured hexahedra; cell (a,b,c) has index a + nx*(b + ny*c).

    Patches, in order: minus_x, plus_x, minus_y, plus_y, minus_z, plus_z (or
    ``names``).  ``warp(points)`` may move the vertices.
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
    return PolyMesh(verts, list(rings), owner, neighbour, patch, list(names), list(kinds))


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


def _circumcentres(p):
    """Circumcentres of tetrahedra p (M,4,3); also |det| of the edge matrix."""
    a = p[:, 0]
    A = p[:, 1:] - a[:, None, :]
    rhs = 0.5 * np.einsum("mij,mij->mi", A, A)
    det = np.linalg.det(A)
    safe = np.abs(det) > 0
    c = np.zeros_like(a)
    c[safe] = a[safe] + np.linalg.solve(A[safe], rhs[safe][:, :, None])[:, :, 0]
    return c, np.abs(det)


def voronoi_cube(n: int, jitter: float = 0.3, seed: int = 20261007, names=None, kinds=None) -> PolyMesh:
    """Voronoi tessellation of the unit cube from a jittered n^3 lattice of sites.

    Site (i,j,k) = ((i,j,k) + 0.5 + U(-jitter, jitter)^3) / n, cell index
    i + n*(j + n*k), seeded by ``seed``.  Sites within 2.5/n of a cube face are
    mirrored across it; the bisector of a site and its own mirror is the cube
    face, so every cell is exactly its Voronoi cell clipped to the cube.  The
    tessellation is the dual of the Delaunay tetrahedralisation (scipy/qhull):
    Voronoi vertices are tetrahedron circumcentres and the face between sites
    i and j is the ring of circumcentres of the tetrahedra around edge (i,j).
    Coincident circumcentres (cospherical site groups, which the mirror planes
    create) are merged at 1e-9/n.  Patches: minus_x, plus_x, minus_y, plus_y,
    minus_z, plus_z.
    """
    from scipy.spatial import Delaunay
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    ii, jj, kk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    lattice = np.stack([ii.ravel(order="F"), jj.ravel(order="F"), kk.ravel(order="F")], axis=1).astype(float)
    sites = (lattice + 0.5 + rng.uniform(-jitter, jitter, size=lattice.shape)) * h
    N = len(sites)
    layer = 2.5 * h
    mirror_pts, mirror_of, mirror_patch = [], [], []
    for axis in range(3):
        for side in range(2):
            sel = np.nonzero(sites[:, axis] < layer)[0] if side == 0 else np.nonzero(sites[:, axis] > 1 - layer)[0]
            q = sites[sel].copy()
            q[:, axis] = -q[:, axis] if side == 0 else 2.0 - q[:, axis]
            mirror_pts.append(q)
            mirror_of.append(sel)
            mirror_patch.append(np.full(len(sel), 2 * axis + side))
    pts = np.concatenate([sites] + mirror_pts)
    of = np.concatenate([np.arange(N)] + mirror_of)          # original site of every point
    ppatch = np.concatenate([np.full(N, -1)] + mirror_patch)  # patch of every mirror point
    tri = Delaunay(pts)
    tets = tri.simplices.astype(np.int64)
    cc, det = _circumcentres(pts[tets])
    good = det > 1e-12 * h ** 3
    # edges of the tetrahedra that produce faces of original cells
    pairs = np.array([(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)])
    ea = tets[:, pairs[:, 0]].ravel()
    eb = tets[:, pairs[:, 1]].ravel()
    et = np.repeat(np.arange(len(tets)), 6)
    lo, hi = np.minimum(ea, eb), np.maximum(ea, eb)
    interior = (hi < N)
    own_mirror = (lo < N) & (hi >= N) & (of[hi] == lo)
    keep = (interior | own_mirror) & good[et]
    lo, hi, et = lo[keep], hi[keep], et[keep]
    key = lo * len(pts) + hi
    # merge coincident circumcentres
    q = np.round(cc / (1e-9 * h)).astype(np.int64)
    _, vid = np.unique(q, axis=0, return_inverse=True)
    vid = vid.ravel()
    # angular order of the ring around each edge
    e = pts[hi] - pts[lo]
    e /= np.linalg.norm(e, axis=1)[:, None]
    ref = np.where((np.abs(e[:, 0]) < 0.9)[:, None], np.array([1.0, 0, 0]), np.array([0, 1.0, 0]))
    u = np.cross(e, ref)
    u /= np.linalg.norm(u, axis=1)[:, None]
    v = np.cross(e, u)
    # The face is convex and lies in the bisector plane, but need not surround the
    # Delaunay edge (non-Gabriel edges): order by angle about the ring's mean point.
    _, grp = np.unique(key, return_inverse=True)
    grp = grp.ravel()
    cnt = np.bincount(grp)
    mean = np.stack([np.bincount(grp, weights=cc[et][:, c]) / cnt for c in range(3)], axis=1)
    r = cc[et] - mean[grp]
    ang = np.arctan2(np.einsum("ij,ij->i", r, v), np.einsum("ij,ij->i", r, u))
    order = np.lexsort((ang, key))
    key, lo, hi, vv = key[order], lo[order], hi[order], vid[et[order]]
    start = np.r_[True, key[1:] != key[:-1]]
    # drop consecutive duplicates inside each ring, then the wrap-around duplicate
    dup = np.r_[False, (vv[1:] == vv[:-1]) & ~start[1:]]
    key, lo, hi, vv, start = key[~dup], lo[~dup], hi[~dup], vv[~dup], start[~dup]
    gid = np.cumsum(start) - 1
    first_pos = np.nonzero(start)[0]
    last_pos = np.r_[first_pos[1:], len(vv)] - 1
    wrap = (vv[last_pos] == vv[first_pos]) & (last_pos > first_pos)
    drop = np.zeros(len(vv), bool)
    drop[last_pos[wrap]] = True
    key, lo, hi, vv, gid = key[~drop], lo[~drop], hi[~drop], vv[~drop], gid[~drop]
    counts = np.bincount(gid, minlength=len(first_pos))
    ok_face = counts >= 3
    ok = ok_face[gid]
    lo, hi, vv, gid = lo[ok], hi[ok], vv[ok], gid[ok]
    fstart = np.r_[True, gid[1:] != gid[:-1]]
    f_lo, f_hi = lo[fstart], hi[fstart]
    sizes = np.diff(np.r_[np.nonzero(fstart)[0], len(vv)])
    # compact vertex numbering
    used, ids = np.unique(vv, return_inverse=True)
    rep = np.zeros(used.max() + 1 if len(used) else 0, np.int64)
    # representative coordinates: the circumcentre of one tetrahedron per merged vertex
    first_tet = np.full(vid.max() + 1, -1, np.int64)
    first_tet[vid[::-1]] = np.arange(len(vid))[::-1]
    verts = cc[first_tet[used]]
    del rep
    is_int = f_hi < N
    owner = f_lo.astype(np.int32)
    neighbour = np.where(is_int, f_hi, -1).astype(np.int32)
    patch = np.where(is_int, -1, ppatch[f_hi]).astype(np.int32)
    # interior faces first, then boundary faces by patch (stable)
    order = np.lexsort((np.arange(len(owner)), patch))
    offsets = np.r_[0, np.cumsum(sizes)].astype(np.int64)
    ring_ids = ids.astype(np.int32)
    new_off = np.r_[0, np.cumsum(sizes[order])].astype(np.int32)
    gather = np.concatenate([np.arange(offsets[f], offsets[f + 1]) for f in order]) if len(order) < 50000 else \
        _ranges(offsets, order)
    names = names or ["minus_x", "plus_x", "minus_y", "plus_y", "minus_z", "plus_z"]
    kinds = kinds or ["wall"] * 6
    return PolyMesh(verts, None, owner[order], neighbour[order], patch[order], list(names), list(kinds),
                    offsets=new_off, ids=ring_ids[gather])


def _ranges(offsets, order):
    """Concatenation of arange(offsets[f], offsets[f+1]) for f in order, vectorised."""
    sizes = (offsets[1:] - offsets[:-1])[order]
    starts = offsets[:-1][order]
    total = int(sizes.sum())
    base = np.repeat(starts - np.r_[0, np.cumsum(sizes)[:-1]], sizes)
    return base + np.arange(total)
