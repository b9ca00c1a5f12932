"""Oracle mesh builder vs the reference builder's own output (golden fixtures)."""
import numpy as np
import pytest

from conftest import load_golden, golden_inputs, golden_patches
from oracle import mesh as om

MESHES = ["quad", "cavity", "tri", "hex", "hybrid"]


@pytest.mark.parametrize("name", MESHES)
def test_oracle_mesh_matches_reference(name):
    d = load_golden("mesh_" + name)
    nodes, cells, bdict, cfl = golden_inputs(d)
    ndim = int(d["ndim"])
    m = om.build(nodes, cells, bdict, ndim=ndim, cell_face_node_list=cfl)
    # connectivity: bit-exact
    np.testing.assert_array_equal(m.owner, d["owner"])
    np.testing.assert_array_equal(m.neighbour, d["neighbour"])
    ref_p = golden_patches(d)
    assert list(m.boundary_patches.keys()) == list(ref_p.keys())
    for k in ref_p:
        np.testing.assert_array_equal(m.boundary_patches[k], ref_p[k])
    kf = d["cell_faces"].shape[1]
    np.testing.assert_array_equal(m.cell_faces[:, :kf], d["cell_faces"])
    # geometry: the reference's own operation order, 1e-14 relative at most
    for a, b in ((m.area, d["area"]), (m.normal, d["normal"]), (m.fcenter, d["fcenter"]),
                 (m.ccenter, d["ccenter"]), (m.volume, d["volume"])):
        np.testing.assert_allclose(a, b, rtol=1e-14, atol=1e-15)
