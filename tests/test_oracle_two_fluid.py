"""The two-fluid oracle (oracle/two_fluid.py) against the reference's own
TwoFluidSolver run (tests/golden/two_fluid.npz): 3 time steps with the 6-equation
energy model on the quad channel and the hybrid hex/tet mesh."""
import numpy as np
import pytest

from conftest import load_golden, golden_inputs
from two_fluid_case import CASES, setup


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("tag,seed", CASES)
def test_oracle_two_fluid_matches_reference(tag, seed):
    from oracle import mesh as om
    from oracle.two_fluid import TwoFluid
    d = load_golden("mesh_" + tag)
    nodes, cells, bdict, cfl = golden_inputs(d)
    m = om.build(nodes, cells, bdict, ndim=int(d["ndim"]), cell_face_node_list=cfl)
    g = load_golden("two_fluid")
    o = TwoFluid(m)

    def set_field(name, arr):
        o.v[name] = np.array(arr, dtype=np.float64)

    setup(o, list(m.boundary_patches), m.ndim, m.n_cells, seed, set_field)
    np.testing.assert_array_equal(o.v["alpha_g"], g[f"{tag}_init_alpha_g"])
    for step in range(3):
        res = o.step()
        assert abs(res - g[f"{tag}_{step}_res"][0]) <= 1e-6 * abs(g[f"{tag}_{step}_res"][0])
        for f in ("alpha_g", "U_l", "U_g", "p", "T_l", "T_g"):
            assert _rel(o.v[f], g[f"{tag}_{step}_{f}"]) < 1e-11, (tag, step, f, _rel(o.v[f], g[f"{tag}_{step}_{f}"]))
