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
