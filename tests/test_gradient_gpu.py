"""Device drop-ins of green_gauss_gradient, least_squares_gradient and
compute_mass_flux (kcfd.gradient) against the reference's own outputs on its
generator meshes (tests/golden/ops_*.npz), called the reference's way: with field
objects carrying .mesh, .values and per-patch .boundary_values."""
import types

import numpy as np
import pytest

from conftest import load_golden, golden_inputs

pytestmark = pytest.mark.gpu
NAMES = ["quad", "tri", "hex", "hybrid"]


def _field(mesh, values, flat_b, ncomp):
    bv, k = {}, 0
    for nm, fids in mesh.boundary_patches.items():
        bv[nm] = flat_b[k:k + len(fids)]
        k += len(fids)
    return types.SimpleNamespace(mesh=mesh, values=values, boundary_values=bv)


@pytest.mark.parametrize("name", NAMES)
def test_gradients_and_mass_flux_match_reference(name):
    from kcfd import mesh as km
    from kcfd.gradient import compute_mass_flux, green_gauss_gradient, least_squares_gradient
    d = load_golden("mesh_" + name)
    nodes, cells, bdict, cfl = golden_inputs(d)
    m = km.build_mesh(nodes, cells, bdict, ndim=int(d["ndim"]), cell_face_node_list=cfl)
    g = load_golden("ops_" + name)
    phi = _field(m, g["phi"], g["phi_b"], 1)
    np.testing.assert_allclose(green_gauss_gradient(phi), g["gg"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(least_squares_gradient(phi), g["lsq"], rtol=1e-11, atol=1e-11)
    U = _field(m, g["U"], g["U_b"], m.ndim)
    np.testing.assert_allclose(compute_mass_flux(U, 1.7, m), g["mflux"], rtol=1e-13, atol=1e-14)
