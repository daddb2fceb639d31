"""Polyhedral mesh geometry, restated from the reference.  TEST INFRASTRUCTURE ONLY.

Follows Mesh::polyhedral (src/core/mesh.cpp:321-564) and its helpers
polygonTriangles / polygonAreaVector / polygonGeometry (src/core/mesh.cpp:60-195),
and the BABELSIM_MESH 3 reader (src/io/mesh_reader.cpp:44-111).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class PolyMesh:
    """Raw polyhedral description: vertices, face rings, owner/neighbour/patch."""
    vertices: np.ndarray                 # (V,3) float64
    faces: list                          # list of int arrays (vertex rings)
    owner: np.ndarray                    # (F,) int32
    neighbour: np.ndarray                # (F,) int32, -1 on boundary
    patch: np.ndarray                    # (F,) int32, -1 on interior faces
    patch_names: list = field(default_factory=list)
    patch_kinds: list = field(default_factory=list)


def read_mesh(path) -> PolyMesh:
    """BABELSIM_MESH 3 reader (src/io/mesh_reader.cpp:44-111)."""
    tokens = open(path).read().split()
    pos = 0

    def take():
        nonlocal pos
        t = tokens[pos]
        pos += 1
        return t
    assert take() == "BABELSIM_MESH" and int(take()) == 3
    assert take() == "vertices"
    nv = int(take())
    verts = np.array(tokens[pos:pos + 3 * nv], dtype=np.float64).reshape(nv, 3)
    pos += 3 * nv
    assert take() == "faces"
    nf = int(take())
    faces, owner, nbr, patch = [], np.empty(nf, np.int32), np.empty(nf, np.int32), np.empty(nf, np.int32)
    for f in range(nf):
        assert take() == "face"
        k = int(take())
        owner[f], nbr[f], patch[f] = int(take()), int(take()), int(take())
        faces.append(np.array(tokens[pos:pos + k], dtype=np.int64))
        pos += k
    assert take() == "patches"
    npatch = int(take())
    names, kinds = [], []
    for _ in range(npatch):
        assert take() == "patch"
        names.append(take())
        kinds.append(take())
    assert take() == "end"
    return PolyMesh(verts, faces, owner, nbr, patch, names, kinds)


def _triangles(ring, verts):
    """polygonTriangles (src/core/mesh.cpp:60-161): fan for convex rings, ear clipping otherwise."""
    p = verts[ring]
    normal = 0.5 * np.cross(p, np.roll(p, -1, axis=0)).sum(axis=0)
    span = p.max(axis=0) - p.min(axis=0)
    a = np.abs(normal)
    drop = (2 if a[2] > a[1] else 1) if a[1] > a[0] else (2 if a[2] > a[0] else 0)
    scale = max(span[0], span[1], span[2], 1.0)
    tol = 1e-13 * scale * scale
    if drop == 0:
        q = p[:, [1, 2]]
    elif drop == 1:
        q = p[:, [2, 0]]
    else:
        q = p[:, [0, 1]]
    nxt = np.roll(q, -1, axis=0)
    signed = float(np.sum(q[:, 0] * nxt[:, 1] - nxt[:, 0] * q[:, 1]))
    if abs(signed) <= tol:
        raise ValueError("polyhedral face projects to zero area")
    orient = 1.0 if signed > 0 else -1.0

    def cross2(a_, b_, c_):
        return (b_[0] - a_[0]) * (c_[1] - a_[1]) - (b_[1] - a_[1]) * (c_[0] - a_[0])
    n = len(ring)
    convex, saw = True, False
    for i in range(n):
        turn = orient * cross2(q[(i - 1) % n], q[i], q[(i + 1) % n])
        saw = saw or abs(turn) > tol
        if turn < -tol:
            convex = False
            break
    if not saw:
        raise ValueError("polyhedral face is collinear")
    if convex:
        return [(ring[0], ring[i], ring[i + 1]) for i in range(1, n - 1)]
    remaining = list(range(n))
    tris = []
    while len(remaining) > 3:
        clipped = False
        m = len(remaining)
        for pos in range(m):
            pv, cu, nx = remaining[(pos - 1) % m], remaining[pos], remaining[(pos + 1) % m]
            if orient * cross2(q[pv], q[cu], q[nx]) <= tol:
                continue
            inside = False
            for c in remaining:
                if c in (pv, cu, nx):
                    continue
                ab = orient * cross2(q[pv], q[cu], q[c])
                bc = orient * cross2(q[cu], q[nx], q[c])
                ca = orient * cross2(q[nx], q[pv], q[c])
                if ab >= -tol and bc >= -tol and ca >= -tol:
                    inside = True
                    break
            if inside:
                continue
            tris.append((ring[pv], ring[cu], ring[nx]))
            remaining.pop(pos)
            clipped = True
            break
        if not clipped:
            raise ValueError("polyhedral face is self-intersecting")
    tris.append((ring[remaining[0]], ring[remaining[1]], ring[remaining[2]]))
    return tris


@dataclass
class Geometry:
    owner: np.ndarray
    neighbour: np.ndarray
    patch: np.ndarray
    Sf: np.ndarray
    xf: np.ndarray
    area: np.ndarray
    normal: np.ndarray
    weight: np.ndarray
    dcoef: np.ndarray
    kvec: np.ndarray
    skew: np.ndarray
    xc: np.ndarray
    volume: np.ndarray
    orthogonal: bool
    patch_names: list
    patch_kinds: list

    @property
    def n_cells(self):
        return len(self.volume)

    @property
    def n_faces(self):
        return len(self.owner)


def compute_geometry(mesh: PolyMesh) -> Geometry:
    """Mesh::polyhedral face/cell geometry (src/core/mesh.cpp:321-564)."""
    verts = mesh.vertices
    nf = len(mesh.faces)
    owner, nbr = mesh.owner.astype(np.int64), mesh.neighbour.astype(np.int64)
    ncell = int(max(owner.max(), nbr.max()) + 1)
    # Orientation reference: mean of all face points of a cell (mesh.cpp:361-377).
    psum = np.zeros((ncell, 3))
    pcnt = np.zeros(ncell)
    for f, ring in enumerate(mesh.faces):
        s = verts[ring].sum(axis=0)
        psum[owner[f]] += s
        pcnt[owner[f]] += len(ring)
        if nbr[f] >= 0:
            psum[nbr[f]] += s
            pcnt[nbr[f]] += len(ring)
    ref = psum / np.maximum(pcnt, 1)[:, None]
    Sf = np.zeros((nf, 3))
    xf = np.zeros((nf, 3))
    area = np.zeros(nf)
    rings, tris_all = [], []
    for f, ring in enumerate(mesh.faces):
        ring = np.asarray(ring)
        tris = _triangles(ring, verts)
        a = sum(0.5 * np.cross(verts[t[1]] - verts[t[0]], verts[t[2]] - verts[t[0]]) for t in tris)
        avg = verts[ring].mean(axis=0)
        if np.dot(a, avg - ref[owner[f]]) < 0.0:
            ring = np.concatenate([ring[:1], ring[1:][::-1]])
            tris = _triangles(ring, verts)
            a = sum(0.5 * np.cross(verts[t[1]] - verts[t[0]], verts[t[2]] - verts[t[0]]) for t in tris)
        c = np.zeros(3)
        tot = 0.0
        for t in tris:
            A, B, C = verts[t[0]], verts[t[1]], verts[t[2]]
            wgt = np.linalg.norm(0.5 * np.cross(B - A, C - A))
            c += wgt * ((A + B + C) / 3.0)
            tot += wgt
        Sf[f], xf[f], area[f] = a, c / tot, tot
        rings.append(ring)
        tris_all.append(tris)
    normal = Sf / area[:, None]
    # Cell volume / centroid from signed tetrahedra about the reference point (mesh.cpp:486-519).
    vol = np.zeros(ncell)
    mom = np.zeros((ncell, 3))
    for f in range(nf):
        for side, cell in ((1.0, owner[f]), (-1.0, nbr[f])):
            if cell < 0:
                continue
            r = ref[cell]
            for t in tris_all[f]:
                A, B, D = verts[t[0]], verts[t[1]], verts[t[2]]
                tet = side * np.dot(A - r, np.cross(B - r, D - r)) / 6.0
                vol[cell] += tet
                mom[cell] += tet * ((r + A + B + D) / 4.0)
    xc = mom / vol[:, None]
    # Face coefficients, weights, skewness (mesh.cpp:521-564).
    interior = nbr >= 0
    delta = np.where(interior[:, None], xc[np.maximum(nbr, 0)] - xc[owner], xf - xc[owner])
    d2 = np.einsum("ij,ij->i", delta, delta)
    proj = np.einsum("ij,ij->i", Sf, delta)
    dcoef = proj / d2
    kvec = Sf - dcoef[:, None] * delta
    orthogonal = bool(np.all(np.linalg.norm(kvec, axis=1) <= 1e-12 * area))
    weight = np.ones(nf)
    skew = np.zeros((nf, 3))
    od = np.abs(np.einsum("ij,ij->i", xf - xc[owner], normal))
    nd = np.abs(np.einsum("ij,ij->i", xc[np.maximum(nbr, 0)] - xf, normal))
    weight[interior] = (nd / (od + nd))[interior]
    denom = np.einsum("ij,ij->i", delta, normal)
    frac = np.einsum("ij,ij->i", xf - xc[owner], normal) / denom
    sk = xf - (xc[owner] + frac[:, None] * delta)
    skew[interior] = sk[interior]
    if np.any(np.linalg.norm(skew[interior], axis=1) > 1e-12 * np.sqrt(d2[interior])):
        orthogonal = False
    return Geometry(owner.astype(np.int32), nbr.astype(np.int32), mesh.patch.astype(np.int32), Sf, xf, area,
                    normal, weight, dcoef, kvec, skew, xc, vol, orthogonal,
                    list(mesh.patch_names), list(mesh.patch_kinds))


def geometry_from_arrays(arrays: dict, patch_names=None, patch_kinds=None) -> Geometry:
    """Build a Geometry from arrays dumped by the reference (oracle/ref/oracle_driver.cpp)."""
    return Geometry(arrays["face_owner"], arrays["face_neighbour"], arrays["face_patch"],
                    arrays["face_area_vectors"], arrays["face_centres"], arrays["face_areas"],
                    arrays["face_normals"], arrays["face_owner_weights"],
                    arrays["face_orthogonal_coefficients"], arrays["face_non_orthogonal"],
                    arrays["face_skewness"], arrays["cell_centres"], arrays["cell_volumes"],
                    bool(arrays["orthogonal_geometry"][0]), list(patch_names or []), list(patch_kinds or []))
