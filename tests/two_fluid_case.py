"""Shared set-up of the two-fluid parity cases, restating make_golden.two_fluid_setup
for the oracle and the device solver (both expose the reference's TwoFluidSolver
set-up methods): inlet / outlet / heated bottom wall / adiabatic walls, seeded
alpha_g in [0.02, 0.08], T_l in [370, 376] K, T_g in [371.15, 375.15] K, 6-equation
energy, dt = 1e-3, 4 inner SIMPLE iterations per step."""
import numpy as np


def setup(sv, patch_names, ndim, n, seed, set_field):
    """set_field(name, array) assigns a cell field on `sv`."""
    rng = np.random.default_rng(seed)
    sv.d_b = 0.003
    sv.solve_energy = True
    sv.max_outer_iter = 4
    sv.tol = 1e-12
    sv.dt = 1e-3
    sv.initialize(0.05)
    ul = [0.1] + [0.0] * (ndim - 1)
    ug = [0.2] + [0.0] * (ndim - 1)
    sv.set_inlet_bc("inlet", 0.05, U_l=ul, U_g=ug, T_l=372.0, T_g=373.0)
    sv.set_outlet_bc("outlet", 0.0)
    for nm in patch_names:
        if nm.startswith("wall"):
            sv.set_wall_bc(nm, q_wall=2.0e4 if nm == "wall_bottom" else None)
    ag = rng.uniform(0.02, 0.08, n)
    set_field("alpha_g", ag.copy())
    set_field("alpha_l", 1.0 - ag)
    set_field("T_l", 370.0 + rng.uniform(0.0, 6.0, n))
    set_field("T_g", 373.15 + rng.uniform(-2.0, 2.0, n))
    set_field("U_l", np.tile(np.array(ul), (n, 1)) * rng.uniform(0.5, 1.5, (n, 1)))
    set_field("U_g", np.tile(np.array(ug), (n, 1)) * rng.uniform(0.5, 1.5, (n, 1)))


CASES = (("quad", 11), ("hybrid", 12))
