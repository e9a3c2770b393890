"""B200 (sm_100a) sparse solve of the profile-curves deformer.

Public surface: `cut_mesh`, `CutMeshSolver`, `solve_multi`,
`solve_deformation` (tool_godot_curvenet_b200.solver), the seeded workload
generators (tool_godot_curvenet_b200.synth) and the C ABI in
include/curvenet_b200.h (tool_godot_curvenet_b200._lib).
"""
from .solver import (BatchSolver, CnError, CutMeshSolver, cut_mesh, lbs_matvec_device,  # noqa: F401
                     solve_deformation, solve_multi)
