"""3D Voronoi tessellation of the unit cube from jittered lattice sites.

Site (i,j,k) = ((i,j,k) + 0.5 + U(-jitter, jitter)^3) / n with a seeded
generator; cell index i + n*(j + n*k).  Sites within 2.5/n of a cube face are
mirrored across it; the bisector of a site and its own mirror is the cube
face, so every cell is exactly its Voronoi cell clipped to the cube.  The
tessellation is the dual of the Delaunay tetrahedralisation (scipy/qhull):
Voronoi vertices are tetrahedron circumcentres and the face between sites i
and j is the ring of circumcentres of the tetrahedra around edge (i,j), ordered
by angle about the ring's mean point in the bisector plane.  Coincident
circumcentres (cospherical site groups, which the mirror planes create) closer
than 1e-9/n are merged.  Everything after the triangulation is vectorised numpy.
"""
from __future__ import annotations

import numpy as np

from .meshgen import PolyMesh

PATCHES = ["minus_x", "plus_x", "minus_y", "plus_y", "minus_z", "plus_z"]


def sites(n: int, jitter: float = 0.3, seed: int = 20261007) -> np.ndarray:
    rng = np.random.default_rng(seed)
    ii, jj, kk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    lattice = np.stack([ii.ravel(order="F"), jj.ravel(order="F"), kk.ravel(order="F")], axis=1).astype(float)
    return (lattice + 0.5 + rng.uniform(-jitter, jitter, size=lattice.shape)) / n


def _circumcentres(p):
    a = p[:, 0]
    A = p[:, 1:] - a[:, None, :]
    rhs = 0.5 * np.einsum("mij,mij->mi", A, A)
    det = np.linalg.det(A)
    safe = np.abs(det) > 0
    c = np.zeros_like(a)
    c[safe] = a[safe] + np.linalg.solve(A[safe], rhs[safe][:, :, None])[:, :, 0]
    return c, np.abs(det)


def _merge_ids(c, good, tol):
    """Vertex ids of the circumcentres: those of `good` tetrahedra closer than `tol` (transitively)
    share an id, every other tetrahedron gets an id of its own.

    Pairs come from a KD-tree and ids are connected components, so two centres
    a rounding error apart always merge (a quantisation grid would split the
    pairs that straddle a grid boundary and leave a non-manifold cell surface).
    """
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    from scipy.spatial import cKDTree
    idx = np.nonzero(good)[0]
    pairs = cKDTree(c[idx]).query_pairs(tol, output_type="ndarray")
    n = len(idx)
    graph = coo_matrix((np.ones(len(pairs), np.int8), (pairs[:, 0], pairs[:, 1])), shape=(n, n))
    n_comp, label = connected_components(graph, directed=False)
    out = np.empty(len(c), np.int64)
    out[idx] = label
    out[~good] = n_comp + np.arange(len(c) - n)
    return out


def _face_areas(ids, sizes, verts):
    off = np.r_[0, np.cumsum(sizes)].astype(np.int64)
    face_of = np.repeat(np.arange(len(sizes)), sizes)
    p = verts[ids]
    p0 = p[off[:-1]][face_of]
    nxt = np.r_[np.arange(1, len(p)), 0]
    nxt[off[1:] - 1] = off[:-1]
    tri = np.cross(p - p0, p[nxt] - p0)
    return 0.5 * np.linalg.norm(np.add.reduceat(tri, off[:-1], axis=0), axis=1)


def _collapse_slivers(ids, sizes, verts, min_area):
    """Collapse faces smaller than `min_area` (near-cospherical site groups) to a point.

    All vertices of a sliver are merged into their mean, every ring is
    re-deduplicated, and rings left with fewer than three vertices disappear.
    Merging keeps every cell a closed, consistently oriented surface (each
    edge still bounds exactly two faces of the cell), which the reference's
    Mesh::validate requires (src/core/mesh.cpp:709-756); the reference also
    rejects faces whose projected area is below 1e-13 (mesh.cpp:89-104).
    Returns (ids, sizes, vertices, kept-face mask over the input faces).
    """
    keep = np.ones(len(sizes), bool)
    verts = verts.copy()
    for _ in range(8):
        area = _face_areas(ids, sizes, verts)
        small = np.nonzero(area <= min_area)[0]
        if len(small) == 0:
            break
        parent = np.arange(len(verts))

        def find(a):
            while parent[a] != a:
                parent[a] = parent[parent[a]]
                a = parent[a]
            return a
        off = np.r_[0, np.cumsum(sizes)]
        for f in small:
            ring = ids[off[f]:off[f + 1]]
            r0 = find(ring[0])
            for v in ring[1:]:
                rv = find(v)
                if rv != r0:
                    parent[rv] = r0
        roots = _roots(parent)
        sums = np.zeros_like(verts)
        np.add.at(sums, roots, verts)
        cnt = np.bincount(roots, minlength=len(verts)).astype(float)
        hit = cnt > 1
        verts[hit] = sums[hit] / cnt[hit][:, None]   # merged vertex at the mean of its members
        ids = roots[ids]
        # de-duplicate consecutive repeats inside rings (and the wrap-around)
        face_of = np.repeat(np.arange(len(sizes)), sizes)
        first = np.r_[True, face_of[1:] != face_of[:-1]]
        dup = np.r_[False, (ids[1:] == ids[:-1]) & ~first[1:]]
        ids, face_of = ids[~dup], face_of[~dup]
        sizes = np.bincount(face_of, minlength=len(sizes))
        off = np.r_[0, np.cumsum(sizes)]
        lastpos = off[1:] - 1
        has = sizes > 1
        wrap = np.zeros(len(ids), bool)
        wrap[lastpos[has]] = ids[lastpos[has]] == ids[off[:-1][has]]
        ids, face_of = ids[~wrap], face_of[~wrap]
        sizes = np.bincount(face_of, minlength=len(sizes))
        alive = sizes >= 3
        if not np.all(alive):
            el = alive[face_of]
            ids = ids[el]
            sizes = sizes[alive]
            idx = np.nonzero(keep)[0]
            keep[idx[~alive]] = False
    return ids, sizes, verts, keep


def _roots(parent):
    r = parent.copy()
    while True:
        nr = r[r]
        if np.array_equal(nr, r):
            return r
        r = nr


def voronoi_cube(n: int, jitter: float = 0.3, seed: int = 20261007, names=None, kinds=None) -> PolyMesh:
    from scipy.spatial import Delaunay
    h = 1.0 / n
    S = sites(n, jitter, seed)
    N = len(S)
    layer = 2.5 * h
    mp, mo, mpatch = [], [], []
    for axis in range(3):
        for side in range(2):
            sel = np.nonzero(S[:, axis] < layer)[0] if side == 0 else np.nonzero(S[:, axis] > 1 - layer)[0]
            q = S[sel].copy()
            q[:, axis] = -q[:, axis] if side == 0 else 2.0 - q[:, axis]
            mp.append(q)
            mo.append(sel)
            mpatch.append(np.full(len(sel), 2 * axis + side))
    pts = np.concatenate([S] + mp)
    of = np.concatenate([np.arange(N)] + mo)
    ppatch = np.concatenate([np.full(N, -1)] + mpatch)
    tets = Delaunay(pts).simplices.astype(np.int64)
    cc, det = _circumcentres(pts[tets])
    good = det > 1e-12 * h ** 3
    vid_of_tet = _merge_ids(cc, good, 1e-9 * h)
    pairs = np.array([(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)])
    ea = tets[:, pairs[:, 0]].ravel()
    eb = tets[:, pairs[:, 1]].ravel()
    et = np.repeat(np.arange(len(tets)), 6)
    lo, hi = np.minimum(ea, eb), np.maximum(ea, eb)
    keep = ((hi < N) | ((lo < N) & (hi >= N) & (of[hi] == lo))) & good[et]
    lo, hi, et = lo[keep], hi[keep], et[keep]
    del ea, eb, keep
    key = lo * len(pts) + hi
    o1 = np.argsort(key, kind="stable")
    key, lo, hi, et = key[o1], lo[o1], hi[o1], et[o1]
    start = np.r_[True, key[1:] != key[:-1]]
    sidx = np.nonzero(start)[0]
    grp = np.cumsum(start) - 1
    cnt = np.diff(np.r_[sidx, len(key)])
    c = cc[et]
    mean = np.add.reduceat(c, sidx, axis=0) / cnt[:, None]
    e = pts[hi[sidx]] - pts[lo[sidx]]
    e /= np.linalg.norm(e, axis=1)[:, None]
    ref = np.where((np.abs(e[:, 0]) < 0.9)[:, None], np.array([1.0, 0, 0]), np.array([0, 1.0, 0]))
    u = np.cross(e, ref)
    u /= np.linalg.norm(u, axis=1)[:, None]
    v = np.cross(e, u)
    r = c - mean[grp]
    ang = np.arctan2(np.einsum("ij,ij->i", r, v[grp]), np.einsum("ij,ij->i", r, u[grp]))
    o2 = np.argsort(grp + (ang + np.pi) * (0.999 / (2 * np.pi)), kind="stable")
    grp, vv = grp[o2], vid_of_tet[et[o2]]
    first = np.r_[True, grp[1:] != grp[:-1]]
    dup = np.r_[False, (vv[1:] == vv[:-1]) & ~first[1:]]
    grp, vv, et2 = grp[~dup], vv[~dup], et[o2][~dup]
    first = np.r_[True, grp[1:] != grp[:-1]]
    fpos = np.nonzero(first)[0]
    lpos = np.r_[fpos[1:], len(vv)] - 1
    wrap = (vv[lpos] == vv[fpos]) & (lpos > fpos)
    drop = np.zeros(len(vv), bool)
    drop[lpos[wrap]] = True
    grp, vv, et2 = grp[~drop], vv[~drop], et2[~drop]
    sizes_all = np.bincount(grp, minlength=len(sidx))
    okf = sizes_all >= 3
    ok = okf[grp]
    grp, vv, et2 = grp[ok], vv[ok], et2[ok]
    faces_g = np.nonzero(okf)[0]
    f_lo, f_hi = lo[sidx[faces_g]], hi[sidx[faces_g]]
    sizes = sizes_all[faces_g]
    used, ids = np.unique(vv, return_inverse=True)
    rep = np.empty(used.max() + 1, np.int64)
    rep[vv] = et2
    verts = cc[rep[used]]
    is_int = f_hi < N
    owner = f_lo.astype(np.int32)
    neighbour = np.where(is_int, f_hi, -1).astype(np.int32)
    patch = np.where(is_int, -1, ppatch[f_hi]).astype(np.int32)
    ids, sizes, verts, keep = _collapse_slivers(ids.ravel(), sizes, verts, max(1e-9 * h * h, 1e-12))
    owner, neighbour, patch = owner[keep], neighbour[keep], patch[keep]
    order = np.argsort(patch, kind="stable")            # interior (-1) first, then by patch
    offsets = np.r_[0, np.cumsum(sizes)].astype(np.int64)
    sz = sizes[order]
    starts = offsets[:-1][order]
    gather = np.repeat(starts - np.r_[0, np.cumsum(sz)[:-1]], sz) + np.arange(int(sz.sum()))
    return PolyMesh(verts, None, owner[order], neighbour[order], patch[order], list(names or PATCHES),
                    list(kinds or ["wall"] * 6), offsets=np.r_[0, np.cumsum(sz)].astype(np.int32),
                    ids=ids.ravel()[gather].astype(np.int32))
