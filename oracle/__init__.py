"""CPU oracle for the K-CFD SIMPLE hot path — TEST INFRASTRUCTURE ONLY.

This package restates, in vectorised FP64 numpy/scipy, the algorithms of the
K-CFD reference (senily0/K-CFD) that the CUDA path in ``k-cfd_b200`` replaces:

* ``oracle.mesh``    face discovery, owner/neighbour, geometry
                     (mesh/mesh_reader.py:66-323) and the structured / jittered /
                     Delaunay generators that feed it (mesh/mesh_generator.py:13-126,
                     266-325; mesh/mesh_generator_3d.py:12-206).
* ``oracle.fvm``     FVMSystem and the face/cell operators (core/fvm_operators.py),
                     Green-Gauss gradient (core/gradient.py:12-48), mass flux and
                     MUSCL deferred correction (core/interpolation.py:17-52,163-303).
* ``oracle.linsolve`` BiCGSTAB in the two stopping semantics the reference uses
                     (core/gpu_solver.py:158-199 and scipy's bicgstab as called from
                     core/linear_solver.py:59), Jacobi (core/preconditioner.py:43-47)
                     and a structural, level-scheduled ILU(0).
* ``oracle.simple``  SIMPLESolver (models/single_phase.py:70-377) plus the
                     extensions the reference lacks (over-relaxed non-orthogonal
                     correction, MUSCL momentum convection) — those extensions have
                     no reference counterpart and their parity is unpinned.

Parity pins: tests/golden/make_golden.py imports the reference itself and writes
golden fixtures; tests/test_oracle_mesh.py, test_oracle_ops.py, test_oracle_simple.py,
test_oracle_two_fluid.py, test_oracle_iluk.py and test_oracle_verification.py check
this package against them.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this package, and only as the checker or the timed CPU baseline. The product
(k-cfd_b200) never imports it.
"""
