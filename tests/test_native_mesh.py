"""Native (C++) mesh builder vs the reference builder's output and the oracle.

Host code only: runs without a GPU."""
import numpy as np
import pytest

from conftest import load_golden, golden_inputs, golden_patches
from kcfd import mesh as km, meshgen
from oracle import mesh as om

MESHES = ["quad", "cavity", "tri", "hex", "hybrid"]


@pytest.mark.parametrize("name", MESHES)
def test_native_builder_matches_reference(name):
    d = load_golden("mesh_" + name)
    nodes, cells, bdict, cfl = golden_inputs(d)
    m = km.build_mesh(nodes, cells, bdict, ndim=int(d["ndim"]), cell_face_node_list=cfl)
    np.testing.assert_array_equal(m.owner, d["owner"])
    np.testing.assert_array_equal(m.neighbour, d["neighbour"])
    ref_p = golden_patches(d)
    assert list(m.boundary_patches.keys()) == list(ref_p.keys())
    for k in ref_p:
        np.testing.assert_array_equal(m.boundary_patches[k], ref_p[k])
    kf = d["cell_faces"].shape[1]
    np.testing.assert_array_equal(m.cell_faces[:, :kf], d["cell_faces"])
    for a, b in ((m.area, d["area"]), (m.normal, d["normal"]), (m.fcenter, d["fcenter"]),
                 (m.ccenter, d["ccenter"]), (m.volume, d["volume"])):
        np.testing.assert_allclose(a, b, rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize("name", MESHES)
def test_pattern_slots_and_colourings(name):
    d = load_golden("mesh_" + name)
    nodes, cells, bdict, cfl = golden_inputs(d)
    m = km.build_mesh(nodes, cells, bdict, ndim=int(d["ndim"]), cell_face_node_list=cfl)
    ref = om.build(nodes, cells, bdict, ndim=int(d["ndim"]), cell_face_node_list=cfl)
    ip, ix = om.csr_pattern(ref)
    np.testing.assert_array_equal(m.indptr, ip)
    np.testing.assert_array_equal(m.indices, ix)
    it = m.neighbour >= 0
    # slot maps point at the right (row, col)
    rows = np.repeat(np.arange(m.n_cells), np.diff(m.indptr))
    np.testing.assert_array_equal(rows[m.slot_on[it]], m.owner[it])
    np.testing.assert_array_equal(m.indices[m.slot_on[it]], m.neighbour[it])
    np.testing.assert_array_equal(rows[m.slot_no[it]], m.neighbour[it])
    np.testing.assert_array_equal(m.indices[m.slot_no[it]], m.owner[it])
    np.testing.assert_array_equal(m.indices[m.diag_slot], np.arange(m.n_cells))
    # face colouring: no two faces of one colour share a cell
    for c in range(m.n_int_colors + m.n_bnd_colors):
        f = np.nonzero(m.face_color == c)[0]
        cellsf = np.concatenate([m.owner[f], m.neighbour[f][m.neighbour[f] >= 0]])
        assert len(np.unique(cellsf)) == len(cellsf), f"colour {c} shares a cell"
    # cell colouring: neighbours differ
    nb = m.indices[rows != m.indices]
    rr = rows[rows != m.indices]
    assert np.all(m.cell_color[nb] != m.cell_color[rr])


def test_structured_hex_colour_counts():
    n, c, f, b = meshgen.hex_box_arrays(1, 1, 1, 6, 5, 4, meshgen.CAVITY_3D_NAMES)
    m = km.build_mesh(n, c, b, ndim=3, cell_face_node_list=f)
    assert m.n_cell_colors == 2          # red-black
    assert m.n_levels == 6 + 5 + 4 - 2   # natural-order wavefronts i+j+k
    assert m.n_internal_faces == 5 * 5 * 4 + 6 * 4 * 4 + 6 * 5 * 3


def test_jittered_hex_matches_oracle():
    n, c, f, b = meshgen.hex_box_arrays(1, 1, 1, 7, 6, 5, meshgen.CAVITY_3D_NAMES)
    n = meshgen.jitter_interior(n, (7, 6, 5), (1 / 7, 1 / 6, 1 / 5), 0.2, seed=0)
    m = km.build_mesh(n, c, b, ndim=3, cell_face_node_list=f)
    ref = om.build_3d(n, c, f, b)
    np.testing.assert_array_equal(m.owner, ref.owner)
    np.testing.assert_array_equal(m.neighbour, ref.neighbour)
    for a, bb in ((m.area, ref.area), (m.normal, ref.normal), (m.ccenter, ref.ccenter), (m.volume, ref.volume)):
        np.testing.assert_allclose(a, bb, rtol=1e-14, atol=1e-16)


def test_delaunay_tri_matches_oracle():
    rng = np.random.default_rng(3)
    pts, cells, bd = meshgen.delaunay_tri_arrays(300, rng)
    m = km.build_mesh(pts, cells, bd)
    ref = om.build_2d(pts, cells, bd)
    np.testing.assert_array_equal(m.owner, ref.owner)
    np.testing.assert_array_equal(m.neighbour, ref.neighbour)
    assert list(m.boundary_patches) == list(ref.boundary_patches)
    np.testing.assert_allclose(m.volume, ref.volume, rtol=1e-14)
    assert m.n_boundary_faces == sum(len(v) for v in bd.values())


def test_bad_input_raises():
    from kcfd._lib import KcfdError
    with pytest.raises(KcfdError):
        km.build_mesh(np.zeros((3, 2)), [np.array([0, 1, 7])], {})


def _same_as_oracle(m, ref, ndim):
    np.testing.assert_array_equal(m.owner, ref.owner)
    np.testing.assert_array_equal(m.neighbour, ref.neighbour)
    assert list(m.boundary_patches) == list(ref.boundary_patches)
    for k in ref.boundary_patches:
        np.testing.assert_array_equal(m.boundary_patches[k], ref.boundary_patches[k])
    for a, b in ((m.area, ref.area), (m.normal, ref.normal), (m.ccenter, ref.ccenter), (m.volume, ref.volume)):
        np.testing.assert_allclose(a, b, rtol=1e-14, atol=1e-16)


def test_fan_many_faces_per_node_matches_oracle():
    """A node shared by 600 edges: its face bucket takes the sorted matching path."""
    K = 300
    th = np.linspace(0, 2 * np.pi, K, endpoint=False)
    nodes = np.vstack([[0.0, 0.0], np.c_[np.cos(th), np.sin(th)]])
    cells = np.array([[0, 1 + i, 1 + (i + 1) % K] for i in range(K)])
    bd = {"rim_even": np.array([[1 + i, 1 + (i + 1) % K] for i in range(0, K, 2)]),
          "rim_odd": np.array([[1 + (i + 1) % K, 1 + i] for i in range(1, K, 2)])}
    m = km.build_mesh(nodes, cells, bd)
    _same_as_oracle(m, om.build_2d(nodes, cells, bd), 2)
    assert m.n_faces == 2 * K and m.n_internal_faces == K


def test_ragged_cells_default_patch_and_untagged_faces():
    """Mixed quads and triangles, a patch literally named 'default' and boundary faces
    that no patch lists (they join 'default' in face order)."""
    nodes, cells, bd = meshgen.quad_box_arrays(0, 0, 1, 1, 23, 17)
    cl = [list(c) for c in cells]
    tri = [[c[0], c[1], c[2]] for c in cl[::5]] + [[c[0], c[2], c[3]] for c in cl[::5]]
    cl = [c for i, c in enumerate(cl) if i % 5] + tri
    names = list(bd)
    bd2 = {names[0]: bd[names[0]], "default": bd[names[1]], names[2]: bd[names[2]]}
    m = km.build_mesh(nodes, cl, bd2)
    ref = om.build_2d(nodes, cl, bd2)
    _same_as_oracle(m, ref, 2)
    assert len(m.boundary_patches["default"]) == len(bd[names[1]]) + len(bd[names[3]])


def test_delaunay_tets_match_oracle():
    rng = np.random.default_rng(5)
    nodes, cells, cf, bd = meshgen.delaunay_tet_arrays((0.2, 0.2, 1.0), 4000, rng)
    m = km.build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf)
    _same_as_oracle(m, om.build_3d(nodes, cells, cf, bd), 3)


def test_face_listed_by_three_cells_takes_the_last_later_cell():
    """Three triangles on one edge (0, 1): owner is the first cell, neighbour the last."""
    nodes = np.array([[0.0, 0.0], [1.0, 0.0], [0.5, 1.0], [0.5, -1.0], [0.5, 2.0]])
    cells = [np.array([0, 1, 2]), np.array([1, 0, 3]), np.array([0, 1, 4])]
    m = km.build_mesh(nodes, cells, {})
    ref = om.build_2d(nodes, cells, {})
    np.testing.assert_array_equal(m.owner, ref.owner)
    np.testing.assert_array_equal(m.neighbour, ref.neighbour)
    f = int(m.cell_faces[0, 0])
    assert m.owner[f] == 0 and m.neighbour[f] == 2


def test_offsets_are_checked():
    from kcfd import _lib
    from kcfd._lib import KcfdError
    import ctypes as C
    L = _lib.lib()
    nodes = np.zeros((4, 2))
    cn = np.array([0, 1, 2, 0, 2, 3], dtype=np.int64)
    h = C.c_void_p()
    for ptr in (np.array([1, 3, 6], dtype=np.int64), np.array([0, 3, 3], dtype=np.int64)):
        rc = L.kcfd_mesh_build(2, 4, _lib.ptr(nodes), 2, _lib.ptr(ptr), _lib.ptr(cn), None, None, None, None,
                               0, None, None, None, C.byref(h))
        assert rc == _lib.BAD_INPUT and "kcfd_mesh_build" in _lib.last_error()
    # a 3D face with five nodes
    n3 = np.random.default_rng(0).random((6, 3))
    with pytest.raises(KcfdError, match="2..4 nodes"):
        km.build_mesh(n3, [np.arange(6)], {}, ndim=3,
                      cell_face_node_list=[[np.array([0, 1, 2, 3, 4]), np.array([0, 1, 5]), np.array([1, 2, 5])]])
