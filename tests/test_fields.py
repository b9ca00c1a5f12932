"""Field containers (kcfd.fields) with the reference's API (core/fields.py), on a fixture
mesh built through the reference's builder signature (build_fvmesh_from_arrays)."""
import numpy as np

from conftest import golden_inputs, load_golden
from kcfd.fields import ScalarField, VectorField
from kcfd.mesh import build_fvmesh_from_arrays


def _mesh():
    d = load_golden("mesh_cavity")
    nodes, cells, bdict, cfl = golden_inputs(d)
    return build_fvmesh_from_arrays(nodes, cells, bdict, cell_zone_map={"fluid": list(range(len(cells)))}, ndim=2)


def test_scalar_field_api():
    m = _mesh()
    assert list(m.cell_zones) == ["fluid"]
    p = ScalarField(m, "p", 1.5)
    assert p.values.shape == (m.n_cells,) and p.mean() == 1.5
    assert set(p.boundary_values) == set(m.boundary_patches)
    p.set_boundary("lid", 2.0)
    p.values[:] = np.arange(m.n_cells)
    q = p.copy()
    p.store_old()
    p.values[0] = -1.0
    assert q.values[0] == 0.0 and p.old_values[0] == 0.0 and p.min() == -1.0
    fid = int(m.boundary_patches["lid"][1])
    assert p.get_face_value(fid) == 2.0
    internal = int(np.flatnonzero(m.neighbour >= 0)[0])
    assert p.get_face_value(internal) == p.values[m.owner[internal]]
    p.set_uniform(3.0)
    assert p.max() == 3.0 and all((v == 3.0).all() for v in p.boundary_values.values())


def test_vector_field_api():
    m = _mesh()
    u = VectorField(m, "U", [1.0])
    assert u.values.shape == (m.n_cells, 2) and (u.y == 0).all() and (u.x == 1).all()
    assert (u.z == 0).all()
    u.set_boundary("lid", [1.0, 0.0])
    u.y = 2.0
    np.testing.assert_allclose(u.magnitude(), np.sqrt(5.0))
    v = u.copy()
    u.set_uniform([0.0, 0.0])
    assert (v.x == 1).all() and (u.values == 0).all()
