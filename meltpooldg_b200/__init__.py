"""B200-native matrix-free heat / advection-diffusion operators (MeltPoolDG's
operator path) behind a C ABI (include/mpdg.h, libmpdg.so)."""
from .operators import (AdvectionDiffusionOperator, HeatDiffuseOperator, LinearSolver,  # noqa: F401
                        LinearSolverData, MappedMesh, Mesh, TwoLevelMesh, box_vertices, boundary_mask)
from ._capi import MpdgError, NoConvergence, kernel_launches  # noqa: F401
from .predictor import LeastSquaresProjection  # noqa: F401

__all__ = ["Mesh", "TwoLevelMesh", "MappedMesh", "HeatDiffuseOperator", "AdvectionDiffusionOperator", "LinearSolver",
           "LinearSolverData", "box_vertices", "boundary_mask", "MpdgError", "NoConvergence",
           "kernel_launches", "LeastSquaresProjection"]
