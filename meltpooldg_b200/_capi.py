"""ctypes binding of libmpdg.so (the C ABI declared in include/mpdg.h).

The library is loaded from this package directory.  A missing or unloadable
library raises at import of the operator classes: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpdg.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "mpdg.h")

# status codes (mirror include/mpdg.h)
OK, ERR_ARG, ERR_CUDA, ERR_ALLOC, ERR_NOT_CONVERGED, ERR_BREAKDOWN, ERR_NAN, ERR_UNSUPPORTED, \
    ERR_BUDGET, ERR_SIZE = 0, -1, -2, -3, -4, -5, -6, -7, -8, -9
OP_HEAT, OP_ADVDIFF = 0, 1
FP64, FP32 = 0, 1
VEL_NONE, VEL_ROTATION, VEL_VORTEX, VEL_CONST, VEL_NODAL = 0, 1, 2, 3, 4
GEOM_AUTO, GEOM_GENERAL = 0, 1
SOLVER_CG, SOLVER_GMRES = 0, 1
PREC_IDENTITY, PREC_JACOBI, PREC_CHEBYSHEV = 0, 1, 2
FIELD_TEMPERATURE, FIELD_TEMPERATURE_OLD, FIELD_HEAVISIDE, FIELD_VELOCITY = 0, 1, 2, 3
MAT_LINEAR, MAT_GAS_LIQUID, MAT_LIQUID_SOLID, MAT_GAS_LIQUID_SOLID = 0, 1, 2, 3
AC_POLY4_BELL, AC_CONSTANT, AC_QLQ = 0, 1, 2

_STATUS_NAMES = {0: "OK", -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_ALLOC", -4: "ERR_NOT_CONVERGED",
                 -5: "ERR_BREAKDOWN", -6: "ERR_NAN", -7: "ERR_UNSUPPORTED", -8: "ERR_BUDGET",
                 -9: "ERR_SIZE"}


class MpdgError(RuntimeError):
    def __init__(self, status, where, msg):
        super().__init__(f"{where}: {_STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class NoConvergence(MpdgError):
    """Counterpart of dealii::SolverControl::NoConvergence (linear_solver.hpp:124-129)."""


class MeshDesc(C.Structure):
    _fields_ = [("dim", C.c_int), ("degree", C.c_int), ("nc", C.c_int * 3),
                ("vertices", C.POINTER(C.c_double)), ("dirichlet_mask", C.POINTER(C.c_uint8)),
                ("geometry", C.c_int)]


class MappedMeshDesc(C.Structure):
    _fields_ = [("degree", C.c_int), ("n_cells", C.c_int64), ("n_dofs", C.c_int64),
                ("cell_vertices", C.POINTER(C.c_double)), ("cell_dofs", C.POINTER(C.c_int64)),
                ("dirichlet_mask", C.POINTER(C.c_uint8)), ("n_constraints", C.c_int64),
                ("constrained_dofs", C.POINTER(C.c_int64)), ("constraint_offsets", C.POINTER(C.c_int64)),
                ("constraint_masters", C.POINTER(C.c_int64)), ("constraint_weights", C.POINTER(C.c_double)),
                ("face_ids", C.POINTER(C.c_int8))]


class OpDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("dt", C.c_double), ("rho_cp", C.c_double), ("k0", C.c_double),
                ("k_alpha", C.c_double), ("full_tangent", C.c_int), ("theta", C.c_double),
                ("diffusivity", C.c_double), ("vel_kind", C.c_int), ("vel_param", C.c_double * 3),
                ("precision_mask", C.c_int), ("robin_alpha", C.c_double),
                ("robin_t_inf", C.c_double), ("robin_faces", C.c_int), ("supg", C.c_int),
                ("supg_coefficient", C.c_double), ("rad_emissivity", C.c_double),
                ("rad_t_inf", C.c_double), ("rad_faces", C.c_int), ("material", C.c_int),
                ("mat_rho", C.c_double * 3), ("mat_cp", C.c_double * 3), ("mat_k", C.c_double * 3),
                ("solidus", C.c_double), ("liquidus", C.c_double), ("two_phase_sharp", C.c_int),
                ("solid_liquid_sharp", C.c_int), ("volume_specific", C.c_int),
                ("latent_heat", C.c_double), ("apparent_capacity", C.c_int)]


class SolverDesc(C.Structure):
    _fields_ = [("solver", C.c_int), ("preconditioner", C.c_int), ("max_iterations", C.c_int),
                ("rel_tolerance", C.c_double), ("abs_tolerance", C.c_double),
                ("gmres_restart", C.c_int), ("chebyshev_degree", C.c_int),
                ("lanczos_steps", C.c_int), ("chebyshev_range", C.c_double),
                ("chebyshev_safety", C.c_double), ("mixed_precision", C.c_int),
                ("inner_tolerance", C.c_double), ("max_outer", C.c_int),
                ("reliable_delta", C.c_double)]


class SolveReport(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("outer_iterations", C.c_int),
                ("operator_applies", C.c_int), ("initial_residual", C.c_double),
                ("final_residual", C.c_double), ("lambda_max", C.c_double), ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Schedule(C.Structure):
    _fields_ = [("slabs", C.c_int), ("l2_evict_first", C.c_int), ("overlap_colours", C.c_int),
                ("cta_cell_groups", C.c_int), ("lane_cells", C.c_int)]


class ProblemDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("degree", C.c_int), ("nc", C.c_int), ("dirichlet", C.c_int),
                ("vel_kind", C.c_int), ("max_iterations", C.c_int), ("dt", C.c_double),
                ("rho_cp", C.c_double), ("k0", C.c_double), ("theta", C.c_double),
                ("diffusivity", C.c_double), ("rel_tolerance", C.c_double),
                ("abs_tolerance", C.c_double), ("rhs_seed", C.c_uint64)]


_lib = None


def header_symbols():
    """Function names declared in include/mpdg.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(mpdg_[a-z0-9_]+)\s*\(", text)))


def lib():
    """The loaded library; raises if it is absent (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libmpdg.so is not built ({LIB_PATH}); run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    vp, dp, fp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float)
    L.mpdg_last_error.restype = C.c_char_p
    L.mpdg_kernel_launches.restype = C.c_int64
    L.mpdg_allocations.restype = C.c_int64
    L.mpdg_mesh_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(vp)]
    L.mpdg_mesh_destroy.argtypes = [vp]
    L.mpdg_mesh_create_two_level.argtypes = [C.POINTER(MeshDesc), C.POINTER(MeshDesc), C.POINTER(vp)]
    L.mpdg_mesh_create_mapped.argtypes = [C.POINTER(MappedMeshDesc), C.POINTER(vp)]
    L.mpdg_mesh_n_dofs.argtypes = [vp, C.POINTER(C.c_int64)]
    L.mpdg_mesh_device_bytes.argtypes = [vp, C.POINTER(C.c_int64)]
    L.mpdg_op_create.argtypes = [vp, C.POINTER(OpDesc), C.POINTER(vp)]
    L.mpdg_op_destroy.argtypes = [vp]
    L.mpdg_op_reset_time_increment.argtypes = [vp, C.c_double]
    L.mpdg_op_use_dirichlet.argtypes = [vp, C.c_int]
    L.mpdg_op_set_field.argtypes = [vp, C.c_int, vp]
    L.mpdg_op_set_stream.argtypes = [vp, vp]
    L.mpdg_op_set_inflow_outflow.argtypes = [vp, C.POINTER(C.c_uint8)]
    L.mpdg_op_set_field_host.argtypes = [vp, C.c_int, dp]
    L.mpdg_compute_inverse_diagonal_host.argtypes = [vp, dp]
    L.mpdg_create_rhs_host.argtypes = [vp, dp, dp, dp]
    L.mpdg_op_device_error.argtypes = [vp, C.POINTER(C.c_int)]
    L.mpdg_debug_set_wait_polls.argtypes = [C.c_int64]
    L.mpdg_vmult.argtypes = [vp, vp, vp]
    L.mpdg_vmult_f32.argtypes = [vp, vp, vp]
    L.mpdg_vmult_multi.argtypes = [vp, C.c_int, C.POINTER(vp), C.POINTER(vp)]
    L.mpdg_fma_peak.argtypes = [dp, dp]
    L.mpdg_op_set_schedule.argtypes = [vp, C.c_int, C.POINTER(Schedule)]
    L.mpdg_op_get_schedule.argtypes = [vp, C.c_int, C.POINTER(Schedule)]
    L.mpdg_op_autotune.argtypes = [vp, C.c_int, C.c_int, C.POINTER(Schedule), dp, dp, C.c_int]
    L.mpdg_vmult_multi_f32.argtypes = [vp, C.c_int, C.POINTER(vp), C.POINTER(vp)]
    L.mpdg_predict_lsq.argtypes = [vp, C.c_int, C.POINTER(vp), vp, vp, C.POINTER(C.c_int)]
    L.mpdg_vmult_host.argtypes = [vp, dp, dp]
    L.mpdg_compute_inverse_diagonal.argtypes = [vp, vp]
    L.mpdg_compute_diagonal.argtypes = [vp, vp]
    L.mpdg_create_rhs.argtypes = [vp, vp, vp, vp]
    L.mpdg_solve.argtypes = [vp, C.POINTER(SolverDesc), vp, vp, C.POINTER(SolveReport)]
    L.mpdg_solve_host.argtypes = [vp, C.POINTER(SolverDesc), dp, dp, C.POINTER(SolveReport)]
    L.mpdg_solver_desc_default.argtypes = [C.POINTER(SolverDesc)]
    L.mpdg_solver_desc_default.restype = None
    L.mpdg_l2_norm.argtypes = [vp, vp, dp]
    L.mpdg_solve_cg_noalloc.argtypes = [vp, vp, vp, C.c_double, C.c_double, C.c_int,
                                        C.POINTER(SolveReport)]
    pd = C.POINTER(ProblemDesc)
    i64p, ip = C.POINTER(C.c_int64), C.POINTER(C.c_int)
    L.mpdg_batch_create.argtypes = [C.c_int64, C.c_int, C.c_double, C.POINTER(vp)]
    L.mpdg_batch_destroy.argtypes = [vp]
    L.mpdg_problem_bytes.argtypes = [pd, i64p, i64p]
    L.mpdg_problem_rhs_host.argtypes = [pd, dp]
    L.mpdg_problem_diagonal_host.argtypes = [pd, dp]
    L.mpdg_batch_submit.argtypes = [vp, pd, dp, i64p]
    L.mpdg_batch_run.argtypes = [vp, C.c_int, C.c_int, ip, ip]
    L.mpdg_batch_poll.argtypes = [vp, C.c_int64, C.POINTER(SolveReport)]
    L.mpdg_batch_take.argtypes = [vp, C.c_int64, dp, C.POINTER(SolveReport)]
    L.mpdg_batch_autotune.argtypes = [vp, ip, dp]
    L.mpdg_batch_shape.argtypes = [vp, ip, ip, ip]
    L.mpdg_batch_used_bytes.argtypes = [vp, i64p]
    L.mpdg_batch_stats.argtypes = [vp, dp, C.c_int]
    L.mpdg_serve.argtypes = [vp, pd, dp, C.c_int, C.c_int, C.POINTER(dp), dp, dp,
                             C.POINTER(SolveReport), dp]
    _lib = L
    return L


def check(status, where):
    if status != OK:
        msg = lib().mpdg_last_error().decode(errors="replace")
        cls = NoConvergence if status == ERR_NOT_CONVERGED else MpdgError
        raise cls(status, where, msg)
    return status


def kernel_launches():
    return int(lib().mpdg_kernel_launches())


def allocations():
    """Device and pinned-host allocations the library has made since load."""
    return int(lib().mpdg_allocations())
