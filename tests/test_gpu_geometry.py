"""Device geometry (Mesh::polyhedral, src/core/mesh.cpp:321-564, on the GPU) against the host geometry.

Bar: every geometry array bit-identical to the host computation (the device
evaluates the same expressions in the same order without FMA contraction),
the orthogonal flag equal, and the error message of every rejected mesh equal
to the host's.  The non-convex block mesh is also checked against the numpy
restatement (1e-12), which is pinned to the reference.
"""
import numpy as np
import pytest

from babelsim_b200 import meshgen
from babelsim_b200.api import validate_polyhedral
from babelsim_b200._lib import BsgError
from helpers import CASES, GEO_KEYS, PISO_CASES, RANS_CASES, Golden
from oracle import geometry

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import babelsim_b200 as bsg
    c = bsg.Context(0)
    yield c
    c.close()


def l_block(reverse=()):
    """Two cells on a 2x2x1 block: an L-shaped cell (three unit squares, non-convex top and bottom
    faces that need ear clipping) and the unit cube in the notch.  Faces listed in `reverse` are
    given with their ring reversed.  The orientation reference of the L cell (the mean of its face
    points) lies on the planes of its two interior faces, so those keep the orientation given
    (outward here; reversing them makes the reference reject the mesh); every other face is
    re-oriented outward whatever its given order."""
    P = {}
    verts = []

    def v(x, y, z):
        if (x, y, z) not in P:
            P[(x, y, z)] = len(verts)
            verts.append((x, y, z))
        return P[(x, y, z)]
    L_ring = [(0, 0), (2, 0), (2, 1), (1, 1), (1, 2), (0, 2)]
    faces, owner, nbr, patch = [], [], [], []

    def face(ring, o, n, p):
        faces.append([v(*q) for q in ring])
        owner.append(o); nbr.append(n); patch.append(p)
    face([(1, 1, 0), (1, 1, 1), (2, 1, 1), (2, 1, 0)], 0, 1, -1)        # y = 1, x in [1, 2] (+y)
    face([(1, 1, 0), (1, 2, 0), (1, 2, 1), (1, 1, 1)], 0, 1, -1)        # x = 1, y in [1, 2] (+x)
    face([(x, y, 0) for x, y in reversed(L_ring)], 0, -1, 0)            # L bottom (outward -z)
    face([(x, y, 1) for x, y in L_ring], 0, -1, 0)                      # L top
    face([(0, 0, 0), (0, 0, 1), (0, 2, 1), (0, 2, 0)], 0, -1, 0)        # x = 0
    face([(0, 0, 0), (2, 0, 0), (2, 0, 1), (0, 0, 1)], 0, -1, 0)        # y = 0
    face([(2, 0, 0), (2, 1, 0), (2, 1, 1), (2, 0, 1)], 0, -1, 0)        # x = 2, y in [0, 1]
    face([(0, 2, 0), (0, 2, 1), (1, 2, 1), (1, 2, 0)], 0, -1, 0)        # y = 2, x in [0, 1]
    face([(1, 1, 0), (1, 2, 0), (2, 2, 0), (2, 1, 0)], 1, -1, 0)        # cube bottom
    face([(1, 1, 1), (2, 1, 1), (2, 2, 1), (1, 2, 1)], 1, -1, 0)        # cube top
    face([(2, 1, 0), (2, 2, 0), (2, 2, 1), (2, 1, 1)], 1, -1, 0)        # x = 2, y in [1, 2]
    face([(1, 2, 0), (1, 2, 1), (2, 2, 1), (2, 2, 0)], 1, -1, 0)        # y = 2, x in [1, 2]
    faces = [list(reversed(f)) if i in reverse else f for i, f in enumerate(faces)]
    return meshgen.PolyMesh(np.array(verts, float), faces, np.array(owner), np.array(nbr), np.array(patch),
                            ["walls"], ["wall"])


def _meshes():
    out = [(name, Golden(name).poly) for name in CASES + PISO_CASES + RANS_CASES]
    out += [("voronoi6", meshgen.voronoi_cube(6)), ("voronoi12", meshgen.voronoi_cube(12)),
            ("warped7", meshgen.warped_box(7)), ("cylinder", meshgen.cylinder_ogrid(48, 12)),
            ("l_block", l_block()), ("l_block_inward", l_block(reverse=(2, 3, 5, 9)))]
    return out


@pytest.mark.parametrize("name,poly", _meshes(), ids=lambda x: x if isinstance(x, str) else "")
def test_device_geometry_is_bit_identical_to_the_host(ctx, name, poly):
    import babelsim_b200 as bsg
    dev = bsg.Mesh.from_polyhedral(ctx, poly)
    host = bsg.Mesh.from_polyhedral(ctx, poly, host_geometry=True)
    assert (dev.n_cells, dev.n_faces, dev.orthogonal) == (host.n_cells, host.n_faces, host.orthogonal)
    for key in (k for k in GEO_KEYS if k != "orthogonal_geometry"):
        a, b = dev.export(key), host.export(key)
        assert np.array_equal(a, b), (name, key, np.abs(a - b).max())
    dev.close()
    host.close()


@pytest.mark.parametrize("reverse", [(), (2, 3, 5, 9)])
def test_nonconvex_block_matches_the_restatement(ctx, reverse):
    import babelsim_b200 as bsg
    poly = l_block(reverse)
    geo = geometry.compute_geometry(geometry.PolyMesh(poly.vertices, poly.faces, poly.owner, poly.neighbour,
                                                      poly.patch, poly.patch_names, poly.patch_kinds))
    m = bsg.Mesh.from_polyhedral(ctx, poly)
    assert abs(m.export("cell_volumes")[0] - 3.0) < 1e-14 and abs(m.export("cell_volumes")[1] - 1.0) < 1e-14
    np.testing.assert_allclose(m.export("cell_volumes"), geo.volume, rtol=1e-12)
    np.testing.assert_allclose(m.export("cell_centres").reshape(-1, 3), geo.xc, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(m.export("face_area_vectors").reshape(-1, 3), geo.Sf, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(m.export("face_centres").reshape(-1, 3), geo.xf, rtol=1e-12, atol=1e-14)
    m.close()


def _broken():
    out = []
    pm = meshgen.cavity_2d(3)
    pm.vertices = pm.vertices.copy()
    ring = pm.faces[0]
    pm.vertices[ring[1]] = pm.vertices[ring[0]]                  # collapsed edge
    out.append(("collapsed_edge", pm))
    pm = meshgen.cavity_2d(3)
    pm.faces = [list(f) for f in pm.faces]
    pm.faces[5] = [pm.faces[5][0], pm.faces[5][1], pm.faces[5][0], pm.faces[5][2]]   # repeated vertex
    out.append(("repeated_vertex", pm))
    pm = meshgen.cavity_2d(3)
    pm.faces = [list(f) for f in pm.faces]
    f = pm.faces[4]
    pm.faces[4] = [f[0], f[2], f[1], f[3]]                       # bow tie
    out.append(("bow_tie", pm))
    pm = l_block()
    keep = [i for i in range(len(pm.faces)) if i != 6]           # open surface: a boundary face missing
    out.append(("open_cell", meshgen.PolyMesh(pm.vertices, [pm.faces[i] for i in keep], pm.owner[keep],
                                              pm.neighbour[keep], pm.patch[keep], pm.patch_names, pm.patch_kinds)))
    pm = l_block()
    extra = pm.faces[6][0]                                       # same point, another vertex id, in one face only
    pm.vertices = np.vstack([pm.vertices, pm.vertices[extra]])
    pm.faces[6] = [len(pm.vertices) - 1 if q == extra else q for q in pm.faces[6]]
    out.append(("split_vertex", pm))
    out.append(("inward_interior_face", l_block(reverse=(0,))))
    return out


@pytest.mark.parametrize("name,poly", _broken(), ids=lambda x: x if isinstance(x, str) else "")
def test_device_geometry_rejects_with_the_host_message(ctx, name, poly):
    import babelsim_b200 as bsg
    with pytest.raises(BsgError) as host:
        validate_polyhedral(poly)
    with pytest.raises(BsgError) as dev:
        bsg.Mesh.from_polyhedral(ctx, poly)
    assert str(dev.value) == str(host.value), name
    assert "accepts" not in str(dev.value)


def test_mesh_from_file_equals_mesh_from_arrays(tmp_path):
    """The native BABELSIM_MESH 3 reader builds the same device mesh as the arrays it read."""
    import babelsim_b200 as bsg
    from babelsim_b200 import meshgen
    pm = meshgen.voronoi_cube(6, 0.3, 3)
    path = tmp_path / "v.mesh"
    meshgen.write_mesh(path, pm)
    ctx = bsg.Context(0)
    a = bsg.Mesh.from_polyhedral(ctx, pm)
    b = bsg.Mesh.from_file(ctx, path)
    assert b.n_cells == a.n_cells and b.patch_names == list(pm.patch_names)
    for key in ("face_area_vectors", "face_centres", "cell_centres", "cell_volumes", "face_skewness"):
        assert np.array_equal(a.export(key), b.export(key)), key
    a.close()
    b.close()
    ctx.close()
