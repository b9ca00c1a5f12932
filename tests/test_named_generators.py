"""The reference's named mesh generators (kcfd.meshgen.generate_*) build the same meshes
as the reference's own functions with the same arguments: connectivity, patches and
geometry of tests/golden/gen_*.npz, written by calling the reference generators."""
import numpy as np
import pytest

from conftest import golden_patches, load_golden
from kcfd import meshgen

CASES = {
    "channel": lambda: meshgen.generate_channel_mesh(1.2, 0.3, 7, 4),
    "cavity": lambda: meshgen.generate_cavity_mesh(0.8, 6),
    "tri_channel": lambda: meshgen.generate_triangle_channel_mesh(1.1, 0.4, 6, 3),
    "bubble_column": lambda: meshgen.generate_bubble_column_mesh(0.15, 0.45, 9, 12),
    "channel_3d": lambda: meshgen.generate_3d_channel_mesh(1.0, 0.5, 0.4, 5, 3, 2),
    "duct_3d": lambda: meshgen.generate_3d_duct_mesh(2.0, 0.3, 0.2, 6, 3, 2),
    "cavity_3d": lambda: meshgen.generate_3d_cavity_mesh(1.0, 0.7, 0.6, 3, 4, 2),
}


@pytest.mark.parametrize("name", list(CASES))
def test_named_generator_matches_reference(name):
    m = CASES[name]()
    d = load_golden("gen_" + name)
    np.testing.assert_array_equal(m.owner, d["owner"])
    np.testing.assert_array_equal(m.neighbour, d["neighbour"])
    ref_p = golden_patches(d)
    assert list(m.boundary_patches) == list(ref_p)
    for k in ref_p:
        np.testing.assert_array_equal(m.boundary_patches[k], ref_p[k])
    for a, b in ((m.area, d["area"]), (m.normal, d["normal"]), (m.ccenter, d["ccenter"]), (m.volume, d["volume"])):
        np.testing.assert_allclose(a, b, rtol=1e-14, atol=1e-15)


def test_hybrid_generator_matches_reference():
    """generate_hybrid_hex_tet_mesh: the reference generator's recorded inputs (nodes,
    cells, per-cell faces, boundary dict) bit for bit, and the built mesh."""
    from conftest import golden_inputs
    d = load_golden("mesh_hybrid")
    nodes, cells, bd, cfl = golden_inputs(d)
    n2, c2, f2, b2 = meshgen.hybrid_hex_tet_arrays(1.0, 0.5, 0.5, 4, 2, 2, 0.5)
    np.testing.assert_array_equal(n2, nodes)
    assert len(c2) == len(cells) and all(np.array_equal(a, b) for a, b in zip(c2, cells))
    assert all(len(a) == len(b) and all(np.array_equal(x, y) for x, y in zip(a, b)) for a, b in zip(f2, cfl))
    assert list(b2) == list(bd)
    for k in bd:
        assert len(b2[k]) == len(bd[k]) and all(np.array_equal(x, y) for x, y in zip(b2[k], bd[k]))
    m = meshgen.generate_hybrid_hex_tet_mesh(1.0, 0.5, 0.5, 4, 2, 2, 0.5)
    np.testing.assert_array_equal(m.owner, d["owner"])
    np.testing.assert_array_equal(m.neighbour, d["neighbour"])
