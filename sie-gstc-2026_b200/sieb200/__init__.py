"""sieb200: B200-native dense method-of-moments hot path of the SIE-GSTC solver.

All compute runs in libsieb200.so (hand-written sm_100a CUDA behind a C ABI,
include/sieb200.h); this package is the host-side mirror of the reference's
solver API. There is no CPU fallback: without a CUDA device the solver calls
raise.
"""

from ._lib import (GSTC, PEC_EFIE, PMCHWT, SOLVER_LU_CUSOLVER, SOLVER_LU_FP64, SOLVER_MIXED_IR,
                   InvalidArgument, SiebError, exported_symbols, lib, library_path)
from .adjoint import (FarFieldConeObjective, cone_directions, far_field_matrix, gstc_solve, omega_records,
                      physical_exterior, tensor_gradient)
from .farfield import (MetasurfaceFarFieldEvaluator, bistatic_rcs, evaluate_surface_integral_fields, far_field,
                       spherical_frames)
from .mesh import MeshData, build_edges, geodesic_sphere, icosphere, infer_sphere_radius, load_obj, make_mesh, \
    revolved_spindle, save_obj
from . import autotune  # noqa: F401
from .solvers import (EXTERIOR, INTERIOR, Context, DenseLuSolver, DielectricOptions,
                      DipoleExcitation, GstcExcitationCase, GstcSieOptions, IsotropicMedium,
                      PecOptions, PlaneWaveExcitation, assemble_matrix, assemble_matrix_device,
                      assemble_rhs, default_context, incident_fields, matvec, matvec_matrix_free,
                      solve_dielectric_dense,
                      solve_gstc_dense, solve_gstc_dense_batch, solve_gstc_sweep_batched, solve_pec_dense,
                      SweepInstance, zgemm)

__all__ = [n for n in dir() if not n.startswith("_")]
