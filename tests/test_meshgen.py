"""Mesh generators and the library's host geometry (no GPU needed)."""
import numpy as np
import pytest

from babelsim_b200 import meshgen
from babelsim_b200.api import validate_polyhedral
from oracle import geometry


def _oracle_geo(pm):
    return geometry.compute_geometry(geometry.PolyMesh(pm.vertices, pm.rings(), pm.owner, pm.neighbour, pm.patch,
                                                       pm.patch_names, pm.patch_kinds))


@pytest.mark.parametrize("n", [6, 12])
def test_voronoi_cube_is_a_closed_tessellation(n):
    pm = meshgen.voronoi_cube(n)
    geo = _oracle_geo(pm)
    assert geo.n_cells == n ** 3
    assert abs(geo.volume.sum() - 1.0) < 1e-12
    closure = np.zeros((geo.n_cells, 3))
    np.add.at(closure, geo.owner, geo.Sf)
    inn = geo.neighbour >= 0
    np.add.at(closure, geo.neighbour[inn], -geo.Sf[inn])
    assert np.abs(closure).max() < 1e-12 / n ** 2 * 100
    faces_per_cell = np.bincount(geo.owner, minlength=geo.n_cells) + np.bincount(geo.neighbour[inn],
                                                                                  minlength=geo.n_cells)
    assert 12.0 < faces_per_cell.mean() < 16.0
    assert not geo.orthogonal
    # the library's host geometry accepts it (the reference's Mesh::polyhedral checks)
    assert validate_polyhedral(pm) == (n ** 3, False)


def test_voronoi_vertex_merge_has_no_grid_boundaries():
    """Circumcentres a rounding error apart merge even where they straddle a multiple of the
    tolerance (the 216000-cell cube had such a pair), and chains merge transitively."""
    from babelsim_b200.voronoi import _merge_ids
    tol = 1e-9
    c = np.array([[0.5 * tol * (1 - 1e-6), 0, 0], [0.5 * tol * (1 + 1e-6), 0, 0], [1.0, 0, 0],
                  [1.0 + 0.9 * tol, 0, 0], [1.0 + 1.8 * tol, 0, 0], [0.5 * tol, 0, 0]])
    good = np.array([True, True, True, True, True, False])
    ids = _merge_ids(c, good, tol)
    assert ids[0] == ids[1] and ids[2] == ids[3] == ids[4] and ids[0] != ids[2]
    assert ids[5] not in ids[:5]


def test_voronoi_cube_216000_cells_is_valid():
    assert validate_polyhedral(meshgen.voronoi_cube(60)) == (216000, False)


def test_voronoi_cube_is_seeded():
    a, b = meshgen.voronoi_cube(5, seed=1), meshgen.voronoi_cube(5, seed=1)
    c = meshgen.voronoi_cube(5, seed=2)
    assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.ids, b.ids)
    assert not np.array_equal(a.vertices, c.vertices)


def test_voronoi_boundary_faces_lie_on_the_cube():
    pm = meshgen.voronoi_cube(8)
    geo = _oracle_geo(pm)
    bf = geo.neighbour < 0
    for patch, (axis, value) in enumerate([(0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (2, 1)]):
        m = bf & (geo.patch == patch)
        assert np.allclose(geo.xf[m, axis], value, atol=1e-12)


def test_mesh_file_round_trip(tmp_path):
    pm = meshgen.voronoi_cube(4)
    meshgen.write_mesh(tmp_path / "v.mesh", pm)
    back = meshgen.read_mesh(tmp_path / "v.mesh")
    assert np.array_equal(back.owner, pm.owner) and np.array_equal(back.neighbour, pm.neighbour)
    assert np.array_equal(np.concatenate(back.faces), pm.ids)
    assert np.allclose(back.vertices, pm.vertices, rtol=0, atol=0)


def test_library_geometry_rejects_what_the_reference_rejects():
    pm = meshgen.cavity_2d(3)
    pm.vertices = pm.vertices.copy()
    ring = pm.faces[0]
    pm.vertices[ring[1]] = pm.vertices[ring[0]]   # collapse an edge of one face: zero-area triangle
    with pytest.raises(Exception):
        validate_polyhedral(pm)


def test_native_mesh_reader_matches_the_python_reader(tmp_path):
    """bsg_mesh_file_info (the native BABELSIM_MESH 3 reader, host only) on files the Python
    writer made and on the reference-format cavity fixture mesh."""
    from babelsim_b200.api import file_info
    for pm in (meshgen.voronoi_cube(5, 0.3, 11), meshgen.cavity_2d(6)):
        path = tmp_path / "m.mesh"
        meshgen.write_mesh(path, pm)
        info = file_info(path)
        assert info["cells"] == pm.n_cells and info["faces"] == len(pm.owner)
        assert info["vertices"] == len(pm.vertices)
        assert [n for n, _ in info["patches"]] == list(pm.patch_names)
        assert [k for _, k in info["patches"]] == list(pm.patch_kinds)


@pytest.mark.parametrize("edit,message", [
    (lambda t: t.replace("BABELSIM_MESH 3", "BABELSIM_MESH 2", 1), "only BABELSIM_MESH version 3 is supported"),
    (lambda t: t.replace("\nend", "\nend extra"), "unexpected trailing token extra"),
    (lambda t: t.replace("minus_x\ngeneric", "minus_x\nplasma"), "unknown patch kind plasma"),
    (lambda t: t.replace("\nfaces\n", "\nfacez\n"), "expected faces"),
    (lambda t: t[:t.index("patches")], "missing patches keyword"),
])
def test_native_mesh_reader_rejects_bad_files_with_the_references_messages(tmp_path, edit, message):
    from babelsim_b200 import BsgError
    from babelsim_b200.api import file_info
    path = tmp_path / "bad.mesh"
    meshgen.write_mesh(path, meshgen.hex_box(2, 2, 2))
    path.write_text(edit(path.read_text()))
    with pytest.raises(BsgError) as err:
        file_info(path)
    assert f"invalid BabelSim mesh file {path}: {message}" in str(err.value)


def shuffled(pm, seed=5):
    """The same mesh with its cells numbered at random (owner / neighbour remapped)."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(pm.n_cells)          # caller cell c -> shuffled number perm[c]
    nb = np.asarray(pm.neighbour)
    own = perm[np.asarray(pm.owner)].astype(np.int32)
    nbr = np.where(nb >= 0, perm[np.maximum(nb, 0)], -1).astype(np.int32)
    off, ids = pm.flat()
    return meshgen.PolyMesh(pm.vertices, None, own, nbr, pm.patch, pm.patch_names, pm.patch_kinds,
                            offsets=off, ids=ids), perm


def test_locality_order_keeps_lattice_meshes_and_reorders_shuffled_ones():
    from babelsim_b200.api import locality_order
    pm = meshgen.voronoi_cube(8, 0.3, 20261007)
    order, applied = locality_order(pm)
    assert not applied and np.array_equal(order, np.arange(pm.n_cells))
    sh, _ = shuffled(pm)
    order, applied = locality_order(sh)
    assert applied and np.array_equal(np.sort(order), np.arange(pm.n_cells))
    pos = np.empty_like(order)
    pos[order] = np.arange(len(order))
    inn = sh.neighbour >= 0
    span = np.abs(pos[sh.owner[inn]] - pos[sh.neighbour[inn]]).mean()
    raw = np.abs(sh.owner[inn] - sh.neighbour[inn]).mean()
    assert span * 3 < raw
    # independent cases concatenated keep their cell ranges
    cat, cells, _ = meshgen.concatenate([sh, meshgen.cavity_2d(5)])
    order, applied = locality_order(cat)
    assert applied
    assert set(order[:cells[1]]) == set(range(cells[1]))
