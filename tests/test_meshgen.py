"""The package's structured generators reproduce the reference generators' arrays."""
import numpy as np

from conftest import load_golden, golden_inputs
from kcfd import meshgen


def _same(bd_a, bd_b):
    assert list(bd_a.keys()) == list(bd_b.keys())
    for k in bd_a:
        np.testing.assert_array_equal(np.asarray(bd_a[k]), np.asarray(bd_b[k]))


def test_quad_channel_arrays():
    nodes, cells, bd, _ = golden_inputs(load_golden("mesh_quad"))
    n2, c2, b2 = meshgen.quad_box_arrays(0.0, 0.0, 1.0, 0.6, 6, 5, meshgen.CHANNEL_2D_NAMES)
    np.testing.assert_array_equal(n2, nodes)
    np.testing.assert_array_equal(c2, np.stack(cells))
    _same(b2, bd)


def test_cavity_arrays():
    nodes, cells, bd, _ = golden_inputs(load_golden("mesh_cavity"))
    n2, c2, b2 = meshgen.quad_box_arrays(0.0, 0.0, 1.0, 1.0, 8, 8, meshgen.CAVITY_2D_NAMES)
    np.testing.assert_array_equal(n2, nodes)
    np.testing.assert_array_equal(c2, np.stack(cells))
    _same(b2, bd)


def test_tri_channel_arrays():
    nodes, cells, bd, _ = golden_inputs(load_golden("mesh_tri"))
    n2, c2, b2 = meshgen.tri_channel_arrays(1.0, 0.5, 5, 3)
    np.testing.assert_array_equal(n2, nodes)
    np.testing.assert_array_equal(c2, np.stack(cells))
    _same(b2, bd)


def test_hex_cavity_arrays():
    nodes, cells, bd, cfl = golden_inputs(load_golden("mesh_hex"))
    n2, c2, f2, b2 = meshgen.hex_box_arrays(1.0, 0.9, 0.8, 4, 3, 2, meshgen.CAVITY_3D_NAMES)
    np.testing.assert_array_equal(n2, nodes)
    np.testing.assert_array_equal(c2, np.stack(cells))
    np.testing.assert_array_equal(f2, np.array([np.stack(f) for f in cfl]))
    _same(b2, bd)


def test_jitter_keeps_boundary_nodes():
    n, c, f, b = meshgen.hex_box_arrays(1, 1, 1, 4, 4, 4)
    j = meshgen.jitter_interior(n, (4, 4, 4), (0.25, 0.25, 0.25), 0.2, seed=0)
    moved = np.any(j != n, axis=1)
    on_b = np.any((n == 0) | (n == 1), axis=1)
    assert not np.any(moved & on_b)
    assert np.count_nonzero(moved) == 27
    assert np.abs(j - n).max() <= 0.2 * 0.25 + 1e-15
