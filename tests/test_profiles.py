"""SIMPLESolver.get_velocity_at_y / get_velocity_at_x (host post-processing) give the
reference's profiles (models/single_phase.py:390-425) on the same U and mesh: the
8x8 cavity after 20 outer iterations, from tests/golden/profiles.npz (written by the
reference's own solver and methods)."""
from types import SimpleNamespace

import numpy as np

from conftest import load_golden
from kcfd import meshgen
from kcfd.simple import SIMPLESolver


def test_profiles_match_reference():
    g = load_golden("profiles")
    sv = object.__new__(SIMPLESolver)        # no device state needed for post-processing
    sv.mesh = meshgen.generate_cavity_mesh(1.0, 8)
    sv.U = SimpleNamespace(values=g["U"])
    for tag, fn, t in (("y05", sv.get_velocity_at_y, 0.5), ("y03", sv.get_velocity_at_y, 0.3),
                       ("x05", sv.get_velocity_at_x, 0.5), ("x09", sv.get_velocity_at_x, 0.9)):
        pos, u, v = fn(t)
        np.testing.assert_array_equal(pos, g[tag + "_pos"])
        np.testing.assert_array_equal(u, g[tag + "_u"])
        np.testing.assert_array_equal(v, g[tag + "_v"])
        assert len(pos) > 0
