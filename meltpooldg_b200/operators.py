"""Host-side mirror of MeltPoolDG's matrix-free operator interface over the
C ABI of libmpdg.so.

Class and method names follow the reference so that code written against
OperatorMatrixFree (include/meltpooldg/core/operator_base.hpp:189-283) reads the
same:

    op = HeatDiffuseOperator(mesh, dt=..., rho_cp=..., k0=...)
    op.vmult(dst, src)                                   # operator_base.hpp:239-243
    op.compute_inverse_diagonal_from_matrixfree(diag)    # operator_base.hpp:268-272
    op.create_rhs(dst, src)                              # operator_base.hpp:208-212
    LinearSolver.solve(op, x, b, LinearSolverData(...))  # linear_solver.hpp:26-134

Vectors are torch tensors on the CUDA device (float64, or float32 for the FP32
form) in the library's lexicographic DoF numbering.  torch only provides device
memory and streams; all arithmetic runs in the library's own kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _capi as A

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the environment
    torch = None


def _dptr(t):
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("vectors must be contiguous CUDA tensors")
    return C.c_void_p(t.data_ptr())


class Mesh:
    """Structured hexahedral mesh with FE_Q(degree) on Gauss-Lobatto points
    (ScratchData + MatrixFree set-up, source/core/scratch_data.cpp:191-268)."""

    def __init__(self, vertices, nc, degree, dirichlet_mask=None, geometry="auto"):
        L = A.lib()
        self.nc = tuple(int(v) for v in nc)
        self.degree = int(degree)
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
        self.mask = None if dirichlet_mask is None else np.ascontiguousarray(dirichlet_mask, np.uint8)
        d = A.MeshDesc(3, self.degree, (C.c_int * 3)(*self.nc),
                       self.vertices.ctypes.data_as(C.POINTER(C.c_double)),
                       None if self.mask is None else self.mask.ctypes.data_as(C.POINTER(C.c_uint8)),
                       A.GEOM_GENERAL if geometry == "general" else A.GEOM_AUTO)
        h = C.c_void_p()
        A.check(L.mpdg_mesh_create(C.byref(d), C.byref(h)), "mpdg_mesh_create")
        self._h = h
        n = C.c_int64()
        L.mpdg_mesh_n_dofs(h, C.byref(n))
        self.n_dofs = int(n.value)
        self.shape = tuple(self.nc[d_] * self.degree + 1 for d_ in range(3))

    @classmethod
    def box(cls, nc, degree, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), perturb=0.0, seed=None,
            dirichlet="none", geometry="auto"):
        V = box_vertices(nc, lo, hi, perturb, seed)
        mask = None
        if dirichlet == "all":
            mask = boundary_mask(nc, degree)
        elif dirichlet is not None and not isinstance(dirichlet, str):
            mask = dirichlet
        return cls(V, nc, degree, mask, geometry)

    def device_bytes(self):
        b = C.c_int64()
        A.lib().mpdg_mesh_device_bytes(self._h, C.byref(b))
        return int(b.value)

    def close(self):
        if getattr(self, "_h", None):
            A.lib().mpdg_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TwoLevelMesh(Mesh):
    """Mesh with hanging nodes (mpdg_mesh_create_two_level): a coarse block
    and a fine block refining it 2:1 in y and z, meeting at the coarse block's
    x = max face; the fine DoFs on that plane hang on the coarse faces.
    Vectors are [coarse block DoFs, fine block DoFs]; the hanging DoFs are
    constrained (kept at 0 in right-hand sides, like Dirichlet DoFs)."""

    def __init__(self, coarse_vertices, nc_coarse, fine_vertices, nc_fine, degree, coarse_mask=None,
                 fine_mask=None, geometry="auto"):
        L = A.lib()
        self.degree = int(degree)
        self.nc_coarse = tuple(int(v) for v in nc_coarse)
        self.nc_fine = tuple(int(v) for v in nc_fine)
        keep = []

        def desc(V, nc, mask):
            V = np.ascontiguousarray(V, dtype=np.float64).reshape(-1, 3)
            m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
            keep.extend([V, m])
            return A.MeshDesc(3, self.degree, (C.c_int * 3)(*nc), V.ctypes.data_as(C.POINTER(C.c_double)),
                              None if m is None else m.ctypes.data_as(C.POINTER(C.c_uint8)),
                              A.GEOM_GENERAL if geometry == "general" else A.GEOM_AUTO)

        dc = desc(coarse_vertices, self.nc_coarse, coarse_mask)
        df = desc(fine_vertices, self.nc_fine, fine_mask)
        h = C.c_void_p()
        A.check(L.mpdg_mesh_create_two_level(C.byref(dc), C.byref(df), C.byref(h)), "mpdg_mesh_create_two_level")
        self._h = h
        n = C.c_int64()
        L.mpdg_mesh_n_dofs(h, C.byref(n))
        self.n_dofs = int(n.value)
        self.n_coarse = int(np.prod([c * self.degree + 1 for c in self.nc_coarse]))
        self.mask = None


class MappedMesh(Mesh):
    """Unstructured hexahedral mesh in the ingestion form
    (mpdg_mesh_create_mapped): each cell's 8 corners (x fastest), its
    (degree+1)^3 global DoFs (lexicographic within the cell), a Dirichlet mask,
    and homogeneous constraints {dof: [(master, weight), ...]} (hanging nodes;
    masters unconstrained).  Vectors use the caller's DoF numbering; the
    constrained DoFs stay 0 in results, like Dirichlet DoFs.  `face_ids`
    (n_cells x 6, -1 interior) gives each cell's local face 2 d + s a boundary
    id 0..5, which the heat operator's robin_faces / rad_faces bits select."""

    def __init__(self, cell_vertices, cell_dofs, n_dofs, degree, dirichlet_mask=None, constraints=None,
                 face_ids=None):
        L = A.lib()
        self.degree = int(degree)
        n3 = (self.degree + 1) ** 3
        self.cell_vertices = np.ascontiguousarray(cell_vertices, np.float64).reshape(-1, 8, 3)
        self.cell_dofs = np.ascontiguousarray(cell_dofs, np.int64).reshape(-1, n3)
        self.n_dofs = int(n_dofs)
        self.mask = None if dirichlet_mask is None else np.ascontiguousarray(dirichlet_mask, np.uint8)
        cons = sorted((int(g), list(ent)) for g, ent in (constraints or {}).items())
        self._cdofs = np.ascontiguousarray([g for g, _ in cons] or [0], np.int64)
        off = np.zeros(len(cons) + 1, np.int64)
        for i, (_, ent) in enumerate(cons):
            off[i + 1] = off[i] + len(ent)
        self._coff = off
        self._cmast = np.ascontiguousarray([m for _, ent in cons for m, _ in ent] or [0], np.int64)
        self._cw = np.ascontiguousarray([w for _, ent in cons for _, w in ent] or [0.0], np.float64)
        self.face_ids = None if face_ids is None else np.ascontiguousarray(face_ids, np.int8).reshape(-1, 6)
        i64 = C.POINTER(C.c_int64)
        d = A.MappedMeshDesc(self.degree, self.cell_dofs.shape[0], self.n_dofs,
                             self.cell_vertices.ctypes.data_as(C.POINTER(C.c_double)),
                             self.cell_dofs.ctypes.data_as(i64),
                             None if self.mask is None else self.mask.ctypes.data_as(C.POINTER(C.c_uint8)),
                             len(cons), self._cdofs.ctypes.data_as(i64), self._coff.ctypes.data_as(i64),
                             self._cmast.ctypes.data_as(i64), self._cw.ctypes.data_as(C.POINTER(C.c_double)),
                             None if self.face_ids is None else self.face_ids.ctypes.data_as(C.POINTER(C.c_int8)))
        h = C.c_void_p()
        A.check(L.mpdg_mesh_create_mapped(C.byref(d), C.byref(h)), "mpdg_mesh_create_mapped")
        self._h = h


def box_vertices(nc, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), perturb=0.0, seed=None):
    """Vertices (x fastest) of an nc[0] x nc[1] x nc[2] box; interior vertices
    displaced by U[-perturb h, perturb h] per coordinate (PCG64(seed))."""
    axes = [np.linspace(lo[d], hi[d], nc[d] + 1) for d in range(3)]
    Z, Y, X = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    V = np.stack([X.reshape(-1), Y.reshape(-1), Z.reshape(-1)], axis=1)
    if perturb > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        h = np.array([(hi[d] - lo[d]) / nc[d] for d in range(3)])
        disp = rng.uniform(-1.0, 1.0, size=V.shape) * perturb * h
        kz, ky, kx = np.meshgrid(np.arange(nc[2] + 1), np.arange(nc[1] + 1), np.arange(nc[0] + 1),
                                 indexing="ij")
        idx = np.stack([kx.reshape(-1), ky.reshape(-1), kz.reshape(-1)], axis=1)
        interior = np.all((idx > 0) & (idx < np.array(nc)), axis=1)
        V[interior] += disp[interior]
    return np.ascontiguousarray(V)


def boundary_mask(nc, degree, faces=None):
    """uint8 mask of the DoFs on the selected box faces ((direction, side) pairs;
    default all six)."""
    shape = tuple(nc[d] * degree + 1 for d in range(3))
    Z, Y, X = np.meshgrid(*[np.arange(s) for s in shape[::-1]], indexing="ij")
    g = [X.reshape(-1), Y.reshape(-1), Z.reshape(-1)]
    m = np.zeros(g[0].shape, dtype=bool)
    for d, s in (faces if faces is not None else [(d, s) for d in range(3) for s in (0, 1)]):
        m |= g[d] == (0 if s == 0 else shape[d] - 1)
    return m.astype(np.uint8)


class _MatrixFreeOperator:
    """Common part of the two operators (OperatorBase + OperatorMatrixFree)."""

    def __init__(self, mesh, desc, precisions):
        mask = 0
        for p in precisions:
            mask |= 1 << (A.FP32 if p in ("fp32", "float32") else A.FP64)
        desc.precision_mask = mask
        h = C.c_void_p()
        A.check(A.lib().mpdg_op_create(mesh._h, C.byref(desc), C.byref(h)), "mpdg_op_create")
        self._h = h
        self.mesh = mesh
        self.n_dofs = mesh.n_dofs
        self._desc = desc
        self._fields = {}

    def vmult_multi(self, dsts, srcs):
        """dsts[v] = A srcs[v] for a list of tensors of one precision, several
        vectors per pass (mpdg_vmult_multi)."""
        if len(dsts) != len(srcs) or not dsts:
            raise ValueError("vmult_multi needs equally many destinations and sources")
        n = len(dsts)
        d = (C.c_void_p * n)(*[t.data_ptr() for t in dsts])
        s = (C.c_void_p * n)(*[t.data_ptr() for t in srcs])
        f = A.lib().mpdg_vmult_multi_f32 if dsts[0].dtype == torch.float32 else A.lib().mpdg_vmult_multi
        A.check(f(self._h, n, d, s), "vmult_multi")

    # OperatorBase::reset_time_increment (operator_base.hpp:41-46)
    def reset_time_increment(self, dt):
        A.check(A.lib().mpdg_op_reset_time_increment(self._h, float(dt)), "reset_time_increment")

    # OperatorBase::reset_dof_index (operator_base.hpp:31-35): with_dirichlet=False
    # selects the constraint set without Dirichlet rows
    def reset_dof_index(self, with_dirichlet=True):
        A.check(A.lib().mpdg_op_use_dirichlet(self._h, int(bool(with_dirichlet))), "reset_dof_index")

    def set_stream(self, stream):
        A.lib().mpdg_op_set_stream(self._h, C.c_void_p(stream.cuda_stream if stream is not None else 0))

    def vmult(self, dst, src):
        if dst.dtype == torch.float32:
            A.check(A.lib().mpdg_vmult_f32(self._h, _dptr(dst), _dptr(src)), "vmult_f32")
        else:
            A.check(A.lib().mpdg_vmult(self._h, _dptr(dst), _dptr(src)), "vmult")

    def vmult_host(self, dst: np.ndarray, src: np.ndarray):
        dp = C.POINTER(C.c_double)
        A.check(A.lib().mpdg_vmult_host(self._h, dst.ctypes.data_as(dp), src.ctypes.data_as(dp)),
                "vmult_host")

    def compute_inverse_diagonal_from_matrixfree(self, diag):
        A.check(A.lib().mpdg_compute_inverse_diagonal(self._h, _dptr(diag)), "compute_inverse_diagonal")

    def compute_diagonal(self, diag):
        A.check(A.lib().mpdg_compute_diagonal(self._h, _dptr(diag)), "compute_diagonal")

    def set_velocity(self, U):
        """The velocity as a DoF vector (operators created with velocity="nodal"):
        a contiguous CUDA float64 tensor of 3 n_dofs values, component-major
        (shape (3, n_dofs) or (3 n_dofs,)) -- the vector the reference operators
        read with read_dof_values_plain (heat_diffuse_operator.cpp:975-980,
        advection_diffusion_operator.cpp:461-465).  Call again after changing
        its values."""
        self._fields["U"] = U
        A.check(A.lib().mpdg_op_set_field(self._h, A.FIELD_VELOCITY, _dptr(U)), "set_field")

    def set_schedule(self, slabs=1, l2_evict_first=False, precision="fp64", overlap_colours=False,
                     cta_cell_groups=False, lane_cells=0):
        """Schedule of the resident apply (mpdg_op_set_schedule): colour launches
        slab by slab over `slabs` z-slabs of cell layers, the L2 evict-first
        hint on the coefficient stream, colour launches that overlap the
        previous colour's tail (programmatic dependent launch), cell groups
        shared by a whole CTA (degrees 2 and 4), and one thread per cell
        (lane_cells 1 or 2: uniform lattices of degree 1 or 2).  Results do not
        depend on it, except for rounding with lane_cells."""
        s = A.Schedule(int(slabs), int(bool(l2_evict_first)), int(bool(overlap_colours)), int(bool(cta_cell_groups)),
                       int(lane_cells))
        A.check(A.lib().mpdg_op_set_schedule(self._h, A.FP32 if precision == "fp32" else A.FP64, C.byref(s)),
                "mpdg_op_set_schedule")

    def schedule(self, precision="fp64"):
        s = A.Schedule()
        A.check(A.lib().mpdg_op_get_schedule(self._h, A.FP32 if precision == "fp32" else A.FP64, C.byref(s)),
                "mpdg_op_get_schedule")
        return {"slabs": s.slabs, "l2_evict_first": bool(s.l2_evict_first),
                "overlap_colours": bool(s.overlap_colours), "cta_cell_groups": bool(s.cta_cell_groups),
                 "lane_cells": s.lane_cells}

    def autotune(self, precision="fp64", reps=10):
        """Times the candidate schedules of the resident apply (mpdg_op_autotune)
        and keeps the fastest; returns (schedule, ms per apply, candidate times)."""
        s = A.Schedule()
        ms = C.c_double()
        cand = (C.c_double * 64)()
        A.check(A.lib().mpdg_op_autotune(self._h, A.FP32 if precision == "fp32" else A.FP64, int(reps),
                                         C.byref(s), C.byref(ms), cand, 64), "mpdg_op_autotune")
        return ({"slabs": s.slabs, "l2_evict_first": bool(s.l2_evict_first),
                 "overlap_colours": bool(s.overlap_colours), "cta_cell_groups": bool(s.cta_cell_groups),
                 "lane_cells": s.lane_cells},
                ms.value, [c for c in cand if c >= 0.0])

    def device_error(self):
        """Reads and clears the device error word (an expired bounded wait)."""
        f = C.c_int()
        A.check(A.lib().mpdg_op_device_error(self._h, C.byref(f)), "device_error")
        return f.value

    def l2_norm(self, u):
        v = C.c_double()
        A.check(A.lib().mpdg_l2_norm(self._h, _dptr(u), C.byref(v)), "l2_norm")
        return v.value

    def close(self):
        if getattr(self, "_h", None):
            A.lib().mpdg_op_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HeatDiffuseOperator(_MatrixFreeOperator):
    """Tangent and residual of the heat equation
    (HeatDiffuseMultiPhaseOperator, source/heat/heat_diffuse_operator.cpp):
    v = rho_cp/dt u + rho_cp vel.grad u, g = k(T) grad u, k(T) = k0 (1 + k_alpha T).
    `full_tangent` adds the Newton term dk/dT grad(T) u (non-symmetric).
    `robin_faces` lists the box faces (direction, side) with the convective
    condition of heat_diffuse_operator.cpp:1088-1129 (tangent alpha u v,
    residual -alpha (T - t_inf) v); `rad_faces` those with the radiative one
    (tangent 4 eps sigma T^3 u v, residual -eps sigma (T^4 - rad_t_inf^4) v).
    `material` selects a phase law (Material, material.templates.hpp:213-760):
    a dict with `kind` ("gas_liquid", "liquid_solid", "gas_liquid_solid"),
    `rho`, `cp`, `k` as (gas, liquid, solid) and `solidus`, `liquidus`,
    `two_phase_sharp`, `solid_liquid_sharp`, `volume_specific`, and for laws
    with a solid phase the latent heat of fusion `latent_heat` with its
    `apparent_capacity` profile ("qlq" by default, "poly4_bell", "constant");
    the laws read the heaviside (`set_heaviside`) and, with a solid phase,
    T_old (`set_temperature_old`)."""

    MATERIALS = {"gas_liquid": A.MAT_GAS_LIQUID, "liquid_solid": A.MAT_LIQUID_SOLID,
                 "gas_liquid_solid": A.MAT_GAS_LIQUID_SOLID}
    APPARENT_CAPACITY = {"poly4_bell": A.AC_POLY4_BELL, "constant": A.AC_CONSTANT, "qlq": A.AC_QLQ}

    def __init__(self, mesh, dt, rho_cp=1.0, k0=1.0, k_alpha=0.0, full_tangent=False,
                 velocity=None, precisions=("fp64",), robin_alpha=0.0, robin_t_inf=0.0,
                 robin_faces=(), rad_emissivity=0.0, rad_t_inf=0.0, rad_faces=(), material=None):
        vk, vp = _velocity(velocity)
        d = A.OpDesc(A.OP_HEAT, dt, rho_cp, k0, k_alpha, int(full_tangent), 0.0, 0.0, vk,
                     (C.c_double * 3)(*vp), 0)
        d.robin_alpha = float(robin_alpha)
        d.robin_t_inf = float(robin_t_inf)
        d.robin_faces = sum(1 << (2 * int(dd) + int(ss)) for dd, ss in robin_faces)
        d.rad_emissivity = float(rad_emissivity)
        d.rad_t_inf = float(rad_t_inf)
        d.rad_faces = sum(1 << (2 * int(dd) + int(ss)) for dd, ss in rad_faces)
        if material:
            kind = material["kind"]
            d.material = self.MATERIALS[kind] if isinstance(kind, str) else int(kind)
            for name in ("rho", "cp", "k"):
                setattr(d, "mat_" + name, (C.c_double * 3)(*[float(v) for v in material.get(name, (0, 0, 0))]))
            d.solidus = float(material.get("solidus", 0.0))
            d.liquidus = float(material.get("liquidus", 0.0))
            d.two_phase_sharp = int(bool(material.get("two_phase_sharp", False)))
            d.solid_liquid_sharp = int(bool(material.get("solid_liquid_sharp", False)))
            d.volume_specific = int(bool(material.get("volume_specific", False)))
            d.latent_heat = float(material.get("latent_heat", 0.0))
            ac = material.get("apparent_capacity", "qlq")
            d.apparent_capacity = self.APPARENT_CAPACITY[ac] if isinstance(ac, str) else int(ac)
        super().__init__(mesh, d, precisions)

    def set_temperature(self, T):
        """The temperature the operator linearises about (the `temperature`
        vector the reference operator holds by reference)."""
        self._fields["T"] = T
        A.check(A.lib().mpdg_op_set_field(self._h, A.FIELD_TEMPERATURE, _dptr(T)), "set_field")

    def set_temperature_old(self, T_old):
        """T_old of the Newton terms of laws with a solid phase (`temperature_old`)."""
        self._fields["T_old"] = T_old
        A.check(A.lib().mpdg_op_set_field(self._h, A.FIELD_TEMPERATURE_OLD, _dptr(T_old)), "set_field")

    def set_heaviside(self, H):
        """The level set as heaviside of the two-phase laws (`level_set_as_heaviside`)."""
        self._fields["H"] = H
        A.check(A.lib().mpdg_op_set_field(self._h, A.FIELD_HEAVISIDE, _dptr(H)), "set_field")

    def create_rhs(self, dst, src, heat_source=None):
        """dst += -R(T): Newton residual with T the operator's temperature and
        src = T_old (heat_diffuse_operator.cpp:783-806)."""
        A.check(A.lib().mpdg_create_rhs(self._h, _dptr(dst), _dptr(src), _dptr(heat_source)), "create_rhs")


class AdvectionDiffusionOperator(_MatrixFreeOperator):
    """theta-scheme advection-diffusion tangent
    (source/level_set/advection_diffusion_operator.cpp): v = u/dt + theta vel.grad u,
    g = theta D grad u.  `supg` adds the SUPG flux tau_K u (u/dt + theta u.grad u
    - theta D lap u) with tau_K = supg_coefficient h_K, or h_K / max_q |u| for a
    negative coefficient (ConvectionStabilizationData, advection_diffusion_operator.cpp:450-533)."""

    def __init__(self, mesh, dt, theta=0.5, diffusivity=0.0, velocity=None,
                 precisions=("fp64",), supg=False, supg_coefficient=-1.0):
        vk, vp = _velocity(velocity)
        d = A.OpDesc(A.OP_ADVDIFF, dt, 0.0, 0.0, 0.0, 0, theta, diffusivity, vk,
                     (C.c_double * 3)(*vp), 0)
        d.supg = int(bool(supg))
        d.supg_coefficient = float(supg_coefficient)
        super().__init__(mesh, d, precisions)

    def set_inflow_outflow(self, mask):
        """Identity rows at the flagged DoFs (set_inflow_outflow_bc +
        do_pre_vmult/do_post_vmult, advection_diffusion_operator.cpp:537-578);
        None clears."""
        if mask is None:
            A.check(A.lib().mpdg_op_set_inflow_outflow(self._h, None), "set_inflow_outflow")
            return
        m = np.ascontiguousarray(mask, np.uint8)
        A.check(A.lib().mpdg_op_set_inflow_outflow(self._h, m.ctypes.data_as(C.POINTER(C.c_uint8))),
                "set_inflow_outflow")

    def create_rhs(self, dst, src):
        """dst += phi_old/dt N - (1-theta) vel.grad phi_old N - (1-theta) D grad phi_old.grad N
        (advection_diffusion_operator.cpp:276-358)."""
        A.check(A.lib().mpdg_create_rhs(self._h, _dptr(dst), _dptr(src), None), "create_rhs")


def _velocity(v):
    if v is None:
        return A.VEL_NONE, (0.0, 0.0, 0.0)
    if isinstance(v, str):
        if v == "vortex":
            return A.VEL_VORTEX, (0.0, 0.0, 0.0)
        if v == "nodal":
            return A.VEL_NODAL, (0.0, 0.0, 0.0)
        raise ValueError(v)
    if isinstance(v, tuple) and v and v[0] == "rotation":
        return A.VEL_ROTATION, (float(v[1]), 0.0, 0.0)
    vals = tuple(float(x) for x in v)
    return A.VEL_CONST, vals


@dataclass
class LinearSolverData:
    """LinearSolverData (include/meltpooldg/linear_algebra/linear_solver_data.hpp:38-51)
    plus the device-only Chebyshev and mixed-precision settings."""
    solver_type: str = "GMRES"
    preconditioner_type: str = "Diagonal"
    max_iterations: int = 10000
    rel_tolerance: float = 1e-12
    abs_tolerance: float = 1e-20
    gmres_restart: int = 30
    chebyshev_degree: int = 5
    lanczos_steps: int = 10
    chebyshev_range: float = 30.0
    chebyshev_safety: float = 1.2
    mixed_precision: bool = False
    inner_tolerance: float = 3e-6
    max_outer: int = 20
    reliable_delta: float = 0.1

    def desc(self):
        d = A.SolverDesc()
        A.lib().mpdg_solver_desc_default(C.byref(d))
        d.solver = A.SOLVER_CG if self.solver_type == "CG" else A.SOLVER_GMRES
        d.preconditioner = {"Identity": A.PREC_IDENTITY, "Diagonal": A.PREC_JACOBI,
                            "Chebyshev": A.PREC_CHEBYSHEV}[self.preconditioner_type]
        d.max_iterations = self.max_iterations
        d.rel_tolerance = self.rel_tolerance
        d.abs_tolerance = self.abs_tolerance
        d.gmres_restart = self.gmres_restart
        d.chebyshev_degree = self.chebyshev_degree
        d.lanczos_steps = self.lanczos_steps
        d.chebyshev_range = self.chebyshev_range
        d.chebyshev_safety = self.chebyshev_safety
        d.mixed_precision = int(self.mixed_precision)
        d.inner_tolerance = self.inner_tolerance
        d.max_outer = self.max_outer
        d.reliable_delta = self.reliable_delta
        return d


class LinearSolver:
    """LinearSolver::solve (include/meltpooldg/linear_algebra/linear_solver.hpp:26-134):
    returns the iteration count, raises NoConvergence when the limit is hit."""

    last_report: dict = {}

    @staticmethod
    def solve(op, solution, rhs, data: LinearSolverData = None):
        data = data or LinearSolverData()
        rep = A.SolveReport()
        st = A.lib().mpdg_solve(op._h, C.byref(data.desc()), _dptr(solution), _dptr(rhs), C.byref(rep))
        LinearSolver.last_report = rep.as_dict()
        A.check(st, "LinearSolver::solve")
        return rep.iterations

    @staticmethod
    def solve_host(op, solution: np.ndarray, rhs: np.ndarray, data: LinearSolverData = None):
        data = data or LinearSolverData()
        rep = A.SolveReport()
        dp = C.POINTER(C.c_double)
        st = A.lib().mpdg_solve_host(op._h, C.byref(data.desc()), solution.ctypes.data_as(dp),
                                     rhs.ctypes.data_as(dp), C.byref(rep))
        LinearSolver.last_report = rep.as_dict()
        A.check(st, "LinearSolver::solve_host")
        return rep.iterations
